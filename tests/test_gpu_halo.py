"""Block halos: the neighbor passes give the same results whether a block's
halo records are staged in shared memory or gathered through the halo list
from global memory, for every block or a mix of both; a halo table that
overflows its capacity is grown and the update redone; the exported
neighbor lists (translated back through the halos) stay exact sets.

SPHGPU_HALO_STAGE sets the staged records per block (0: none staged) and
SPHGPU_HALO_CAPACITY the initial halo table capacity; both are read when a
system is created.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def A():
    from sphgpu import _capi
    _capi.load()
    return _capi


def _run(A, sc, steps, env, fields=None):
    from sphgpu import scenes
    old = {k: os.environ.get(k) for k in env}
    os.environ.update({k: str(v) for k, v in env.items()})
    try:
        g = scenes.build_system(sc, fields=fields)
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    g.step_forward_in_time(steps)
    out = {f: g.download(f) for f in (A.FIELD_POSITION, A.FIELD_VELOCITY, A.FIELD_VOLUME, A.FIELD_PRESSURE)}
    off, idx = g.fluid_neighbors()
    out["nbr"] = (off, idx)
    out["iters"] = g.step_stats()["solver_iterations"]
    g.close()
    return out


def _same(a, b):
    for k, v in a.items():
        if k == "nbr":
            assert np.array_equal(v[0], b[k][0]) and np.array_equal(v[1], b[k][1])
        elif k == "iters":
            assert v == b[k]
        else:
            assert np.array_equal(v, b[k]), k


def test_staged_unstaged_and_mixed_halos_agree_sesph(A):
    from sphgpu import scenes
    sc = scenes.dam_break_sesph_8k()
    ref = _run(A, sc, 20, {})
    _same(ref, _run(A, sc, 20, {"SPHGPU_HALO_STAGE": 0}))
    _same(ref, _run(A, sc, 20, {"SPHGPU_HALO_STAGE": 700}))


def test_staged_unstaged_and_mixed_halos_agree_iisph_volume_map(A):
    from sphgpu import scenes
    from sphgpu.fields import build_volume_map_fields
    sc = scenes.dam_break_iisph_box(n_side=14, spacing=0.02, box=(0.6, 0.32, 0.32))
    sc.parameters = dict(sc.parameters, max_solver_iterations=40)
    verts, faces = sc.mesh
    fields = build_volume_map_fields(verts, faces, 0.08, 0.04)
    ref = _run(A, sc, 8, {}, fields)
    _same(ref, _run(A, sc, 8, {"SPHGPU_HALO_STAGE": 0}, fields))
    _same(ref, _run(A, sc, 8, {"SPHGPU_HALO_STAGE": 700}, fields))


def test_halo_table_overflow_grows_and_redoes_the_update(A):
    from sphgpu import scenes
    sc = scenes.serving_dam_break(20000, "IISPH", seed=7)
    ref = _run(A, sc, 10, {})
    _same(ref, _run(A, sc, 10, {"SPHGPU_HALO_CAPACITY": 256}))
