"""The host's mesh transform (sphgpu.scenes.transform_mesh, euler_to_matrix),
which places container and body meshes before they are sampled or turned into
volume-map fields, against the reference's transform tests
(simulation_lib/tests/utilities/triangle_mesh.rs:327-560: MeshContainer::transform
and build_transform, scale then rotate then translate, nalgebra's
from_euler_angles(roll, pitch, yaw) in degrees).
"""
import math

import numpy as np
import pytest

TRI = np.array([[0.0, 0, 0], [1.0, 0, 0], [0.0, 1, 0]])


@pytest.fixture(scope="module")
def S():
    from sphgpu import scenes
    return scenes


def _rot(axis, a):
    c, s = math.cos(a), math.sin(a)
    if axis == 0:
        return np.array([[1, 0, 0], [0, c, -s], [0, s, c]])
    if axis == 1:
        return np.array([[c, 0, s], [0, 1, 0], [-s, 0, c]])
    return np.array([[c, -s, 0], [s, c, 0], [0, 0, 1]])


def test_pure_translation_shifts_all_positions(S):
    v = S.transform_mesh(TRI, translation=(1, 2, 3))
    assert np.array_equal(v, [[1, 2, 3], [2, 2, 3], [1, 3, 3]])


def test_pure_scale_scales_from_the_origin(S):
    v = S.transform_mesh(TRI, scale=(2, 3, 4))
    assert np.array_equal(v[1], [2, 0, 0]) and np.array_equal(v[2], [0, 3, 0])
    assert np.allclose(S.transform_mesh([[1.0, 1, 1]], scale=(2, 3, 4)), [[2, 3, 4]], atol=1e-12)


def test_identity_parameters_leave_positions_unchanged(S):
    assert np.array_equal(S.transform_mesh(TRI), TRI)


def test_transforms_compose_sequentially_on_current_positions(S):
    v = S.transform_mesh(S.transform_mesh(TRI, translation=(1, 0, 0)), translation=(0, 2, 0))
    assert np.array_equal(v[0], [1, 2, 0])


def test_rotation_is_proper_and_rigid(S):
    v = S.transform_mesh(np.eye(3), rotation_euler_deg=(15, 30, 45)) - S.transform_mesh([[0.0, 0, 0]],
                                                                                        rotation_euler_deg=(15, 30, 45))
    vx, vy, vz = v
    for a in (vx, vy, vz):
        assert abs(np.linalg.norm(a) - 1) < 1e-9
    assert abs(vx @ vy) < 1e-9 and abs(vy @ vz) < 1e-9 and abs(vx @ vz) < 1e-9
    assert abs(np.cross(vx, vy) @ vz - 1) < 1e-9  # right-handed, no reflection


@pytest.mark.parametrize("t, r, s", [((1, 2, -3), (10, 20, 30), (1.5, 0.5, 2.0)),
                                     ((1, -2, 0.5), (15, 30, 45), (1.5, 0.5, 2.0))])
def test_composition_is_scale_then_rotate_then_translate(S, t, r, s):
    roll, pitch, yaw = (math.radians(a) for a in r)
    R = _rot(2, yaw) @ _rot(1, pitch) @ _rot(0, roll)  # from_euler_angles(roll, pitch, yaw)
    pts = np.array([[0.3, -0.7, 1.1], [1.0, 0, 0], [0, 0, 0], [-2.0, 0.5, 0.25]])
    want = (R @ (pts * np.array(s)).T).T + np.array(t)
    assert np.allclose(S.transform_mesh(pts, t, r, s), want, rtol=0, atol=1e-9)
