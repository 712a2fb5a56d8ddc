"""The oracle's fluid surface reconstruction (Fluid::reconstruct_surfaces,
simulation_lib/src/sph/fluid.rs:212-347, around splashsurf_lib 0.14.1).

The reference pins only its empty-input case (tests/sph/fluid.rs:615-624);
the third-party reconstruction itself has no vectors here. These tests hold
the restatement to what a marching-cubes surface of the 0.6 level set must
be: closed and consistently oriented (every directed edge has exactly one
opposite), outward unit normals, an enclosed volume close to the fluid's,
one mesh per fluid id in ascending order, and a lattice aligned to
multiples of the cube size.
"""
from collections import Counter

import numpy as np

SPACING = 0.02
RV = SPACING * SPACING * SPACING
H = 2 * SPACING


def _block(counts, origin, seed):
    from sphgpu import scenes
    return scenes.lattice_block(counts, SPACING, origin=origin, jitter=0.01, seed=seed)


def check_closed_and_outward(P, I, center):
    T = np.asarray(I).reshape(-1, 3)
    directed = Counter()
    for a, b, c in T:
        for u, v in ((a, b), (b, c), (c, a)):
            directed[(u, v)] += 1
    assert all(k == 1 and directed.get((v, u), 0) == 1 for (u, v), k in directed.items())
    fn = np.cross(P[T[:, 1]] - P[T[:, 0]], P[T[:, 2]] - P[T[:, 0]])
    assert np.all(np.einsum("ij,ij->i", fn, P[T].mean(1) - center) > 0)
    return np.einsum("ij,ij->i", P[T[:, 0]], np.cross(P[T[:, 1]], P[T[:, 2]])).sum() / 6.0


def test_empty_fluid_has_no_surfaces(oracle):
    assert oracle.reconstruct_surfaces(np.zeros((0, 3)), np.zeros(0, np.uint32), np.zeros(0), SPACING, RV, H) == []


def test_block_surface_is_closed_outward_and_encloses_the_fluid(oracle):
    pos = _block((10, 10, 10), (0.0, 0.0, 0.0), 1)
    meshes = oracle.reconstruct_surfaces(pos, np.zeros(len(pos), np.uint32), np.full(len(pos), 1000 * RV),
                                         SPACING, RV, H)
    assert len(meshes) == 1
    fid, P, N, I = meshes[0]
    vol = check_closed_and_outward(P, I, pos.mean(0))
    assert abs(vol - (10 * SPACING) ** 3) < 0.05 * (10 * SPACING) ** 3
    assert np.allclose(np.linalg.norm(N, axis=1), 1.0)


def test_one_mesh_per_fluid_id_in_ascending_order(oracle):
    a = _block((6, 6, 6), (0.0, 0.0, 0.0), 2)
    b = _block((5, 5, 5), (0.3, 0.0, 0.0), 3)
    pos = np.concatenate([b, a])
    ids = np.concatenate([np.full(len(b), 7, np.uint32), np.full(len(a), 2, np.uint32)])
    mass = np.concatenate([np.full(len(b), 500 * RV), np.full(len(a), 1000 * RV)])
    meshes = oracle.reconstruct_surfaces(pos, ids, mass, SPACING, RV, H)
    assert [m[0] for m in meshes] == [2, 7]
    for (fid, P, N, I), blk in zip(meshes, (a, b)):
        check_closed_and_outward(P, I, blk.mean(0))
        # the level set is mass-independent: m / rho_i does not depend on m
        assert P[:, 0].min() > blk[:, 0].min() - 2 * SPACING and P[:, 0].max() < blk[:, 0].max() + 2 * SPACING


def test_lattice_is_aligned_to_the_cube_size(oracle):
    pos = _block((4, 4, 4), (0.013, -0.2, 0.7), 4)
    cube = 0.75 * 0.5 * SPACING
    k0, n = oracle.surface_grid(pos, H, cube)
    lo, hi = pos.min(0), pos.max(0)
    for d in range(3):
        assert k0[d] == np.floor((lo[d] - H) / cube) - 1
        assert k0[d] + n[d] - 1 == np.floor((hi[d] + H) / cube) + 1
