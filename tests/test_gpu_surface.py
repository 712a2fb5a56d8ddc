"""Fluid surface reconstruction on the device (sph_reconstruct_surfaces)
against the oracle's restatement (Fluid::reconstruct_surfaces,
simulation_lib/src/sph/fluid.rs:212-347).

Both build the same lattice from the same particle positions (the engine's
state, read back exactly), decide inside/outside from f64 sums and number
vertices by lattice edge and triangles by cell, so the meshes have the same
topology: identical index arrays, vertex positions and normals to 1e-9.
The TriangleMesh recording frame carries these meshes (normals, summed with
atomics, to rounding).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SPACING = 0.02


@pytest.fixture(scope="module")
def A():
    from sphgpu import _capi
    _capi.load()
    return _capi


def _scene():
    from sphgpu import scenes
    sc = scenes.dam_break_sesph_8k(n_side=12)
    right = sc.position[:, 0] > np.median(sc.position[:, 0])
    sc.fluid_id = np.where(right, 3, 0).astype(np.uint32)
    sc.mass = np.where(right, 500.0, 1000.0) * SPACING ** 3
    return sc


def _oracle_meshes(oracle, A, g):
    pos = g.download(A.FIELD_POSITION)
    return oracle.reconstruct_surfaces(pos, g.get_fluid_ids(), g.download(A.FIELD_MASS), SPACING,
                                       SPACING * SPACING * SPACING, 2 * SPACING)


def _compare(gm, om):
    assert [m[0] for m in gm] == [m[0] for m in om]
    for (gid, v, idx), (oid, P, N, I) in zip(gm, om):
        assert np.array_equal(idx, I)
        assert np.allclose(v[:, :3], P, rtol=0, atol=1e-9)
        assert np.allclose(v[:, 3:], N, rtol=0, atol=1e-9)


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_meshes_equal_the_oracle(A, oracle, precision):
    from sphgpu import scenes
    g = scenes.build_system(_scene(), precision=precision)
    gm = g.reconstruct_surfaces()
    assert len(gm) == 2 and all(len(m[2]) > 0 for m in gm)
    _compare(gm, _oracle_meshes(oracle, A, g))
    g.step_forward_in_time(25)
    _compare(g.reconstruct_surfaces(), _oracle_meshes(oracle, A, g))
    g.close()


def test_triangle_mesh_frame_carries_the_meshes(A):
    from sphgpu import scenes
    from test_formats import _Reader
    g = scenes.build_system(_scene())
    g.step_forward_in_time(5)
    frame = g.encode_time_step_info("triangle_mesh", "id")
    meshes = g.reconstruct_surfaces()
    r = _Reader(frame)
    assert r.varint() == 5
    r.i += 12 * 8
    r.varint()  # solver iterations
    r.i += 3 * 8
    assert r.varint() == 0  # FluidVisualization::TriangleMesh
    assert r.varint() == len(meshes)
    for fid, v, idx in meshes:
        assert r.varint() == fid
        nv = r.varint()
        assert nv == len(v)
        got = np.frombuffer(frame[r.i:r.i + 48 * nv], "<f8").reshape(nv, 6)
        r.i += 48 * nv
        assert np.array_equal(got[:, :3], v[:, :3])
        # normals sum face contributions with atomics: equal to rounding
        assert np.allclose(got[:, 3:], v[:, 3:], rtol=0, atol=1e-12)
        assert np.array_equal(np.array(r.vec(r.varint), np.uint32), idx)
    assert r.varint() == 3  # max fluid id
    assert r.varint() == 1  # FluidMeshColoring::FluidId
    assert r.varint() == 1  # BoundaryVisualization::Samples
    g.close()
