"""Launch tuning of the neighbor passes (sph_get_tuning, sph_set_tuning,
sph_autotune): every candidate leaves the results bit for bit unchanged, the
autotuner applies its pick without advancing the system, clones inherit the
tuning, and tunings that do not fit are refused.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def A():
    from sphgpu import _capi
    _capi.load()
    return _capi


@pytest.fixture(scope="module")
def case():
    from sphgpu import scenes
    from sphgpu.fields import build_volume_map_fields
    sc = scenes.dam_break_iisph_box(n_side=12, spacing=0.02, box=(0.6, 0.32, 0.32))
    sc.cfl_time_step = False
    sc.parameters = dict(sc.parameters, max_solver_iterations=30, time_increment=1e-3)
    verts, faces = sc.mesh
    return sc, build_volume_map_fields(verts, faces, 0.08, 0.04)


def _fields(A, g):
    return [g.download(f) for f in (A.FIELD_POSITION, A.FIELD_VELOCITY, A.FIELD_PRESSURE)]


@pytest.mark.parametrize("graphs", [0, 4])
def test_every_tuning_gives_identical_results(A, case, graphs):
    from sphgpu import scenes
    sc, fields = case
    ref = scenes.build_system(sc, fields=fields)
    ref.set_step_graphs(graphs)
    ref.step_forward_in_time(10)
    want = _fields(A, ref)
    ref.close()
    for gb, hs, ss in ((8, 1536, 1536), (4, 0, 0), (8, 1024, 3072), (4, 2048, 256)):
        g = scenes.build_system(sc, fields=fields)
        g.set_tuning(gb, hs, ss)
        g.set_step_graphs(graphs)
        assert g.tuning() == {"gather_batch": gb, "halo_stage": hs, "sweep_stage": ss}
        g.step_forward_in_time(10)
        for got, w in zip(_fields(A, g), want):
            assert np.array_equal(got, w), (gb, hs, ss)
        g.close()


def test_autotune_applies_its_pick_without_stepping(A, case):
    from sphgpu import scenes
    sc, fields = case
    g = scenes.build_system(sc, fields=fields)
    g.step_forward_in_time(2)
    before = _fields(A, g)
    t = g.autotune(steps=3)
    assert t["gather_batch"] in (4, 8) and t["halo_stage"] in (1024, 1536, 2048) and t["ms_per_step"] > 0
    assert t["sweep_stage"] in (1536, 1792, 2048)
    assert g.tuning() == {k: t[k] for k in ("gather_batch", "halo_stage", "sweep_stage")}
    assert g.time_steps_propagated() == 2
    for got, w in zip(_fields(A, g), before):
        assert np.array_equal(got, w)
    c = g.clone()
    assert c.tuning() == g.tuning()
    ref = scenes.build_system(sc, fields=fields)
    ref.step_forward_in_time(2)
    g.step_forward_in_time(5)
    c.step_forward_in_time(5)
    ref.step_forward_in_time(5)
    for a, b, r in zip(_fields(A, g), _fields(A, c), _fields(A, ref)):
        assert np.array_equal(a, r) and np.array_equal(b, r)
    for s in (g, c, ref):
        s.close()


def test_tunings_that_do_not_fit_are_refused(A):
    from sphgpu import scenes
    g = scenes.build_system(scenes.dam_break_sesph_8k(n_side=8))
    before = g.tuning()
    for gb, hs, ss in ((5, 1024, 1536), (4, 100000, 1536), (8, 7000, 1536), (4, 1024, 10000)):
        with pytest.raises(A.SPHError) as e:
            g.set_tuning(gb, hs, ss)
        assert e.value.code == A.SPH_ERR_INVALID
    assert g.tuning() == before
    g.close()
