"""The host's boundary-sample rasteriser (sphgpu.scenes.sample_triangle_surface
and sample_triangle_mesh_surface, which make the StaticSampleBoundary samples
the engine receives) against the reference's sampling tests
(simulation_lib/src/utilities/sampling.rs:267-370 and
tests/utilities/sampling.rs:105-166), with the same triangles, cube, spacings
and tolerances.
"""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def S():
    from sphgpu import scenes
    return scenes


def _tri(S, v0, v1, v2, spacing):
    return S.sample_triangle_surface(np.array(v0, float), np.array(v1, float), np.array(v2, float), spacing)


def _cube(S, spacing):
    return S.sample_triangle_mesh_surface(S.CUBE_VERTICES, S.CUBE_FACES_OUTWARD, spacing)


def test_degenerate_triangles_give_no_samples(S):
    assert len(_tri(S, (0, 0, 0), (0, 0, 0), (0, 1, 0), 0.1)) == 0
    assert len(_tri(S, (0, 0, 0), (1, 0, 0), (2, 0, 0), 0.1)) == 0


def test_right_triangle_matches_the_expected_grid(S):
    pts = _tri(S, (0, 0, 0), (1, 0, 0), (0, 1, 0), 0.5)
    want = [(0, 0, 0), (0.5, 0, 0), (1, 0, 0), (0, 0.5, 0), (0.5, 0.5, 0), (0, 1, 0)]
    assert len(pts) == len(want)
    for e in want:
        assert np.min(np.linalg.norm(pts - np.array(e), axis=1)) < 1e-9, e


def test_samples_lie_in_the_plane_of_an_obtuse_triangle(S):
    v0, v1, v2 = np.array([1.0, 1, 1]), np.array([3.0, 1, 2]), np.array([-2.0, 3, 0.5])
    n = np.cross(v1 - v0, v2 - v0)
    n /= np.linalg.norm(n)
    pts = _tri(S, v0, v1, v2, 0.3)
    assert len(pts) > 0 and np.all(np.abs((pts - v0) @ n) < 1e-9)


def test_finer_spacing_yields_more_samples(S):
    assert len(_tri(S, (0, 0, 0), (2, 0, 0), (0, 2, 0), 0.25)) > len(_tri(S, (0, 0, 0), (2, 0, 0), (0, 2, 0), 1.0))
    assert len(_cube(S, 0.2)) > len(_cube(S, 0.6))


def test_mesh_of_one_triangle_equals_the_direct_call(S):
    v = np.array([[0.0, 0, 0], [1.0, 0, 0], [0.0, 1, 0]])
    via_mesh = S.sample_triangle_mesh_surface(v, np.array([[0, 1, 2]], np.uint32), 0.4)
    assert np.array_equal(via_mesh, _tri(S, v[0], v[1], v[2], 0.4))


def test_cube_samples_lie_on_the_surface_and_cover_several_faces(S):
    assert len(_cube(S, 0.5)) > 0
    pts = _cube(S, 0.4)
    assert np.all(np.abs(np.abs(pts).max(axis=1) - 1.0) < 1e-9)
    pts = _cube(S, 0.5)
    for axis, value in ((0, 1.0), (0, -1.0), (1, 1.0)):
        assert np.any(np.abs(pts[:, axis] - value) < 1e-9), (axis, value)


def test_sampling_is_deterministic(S):
    assert np.array_equal(_cube(S, 0.35), _cube(S, 0.35))
