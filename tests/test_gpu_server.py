"""Scene server (sph_server_*): continuous batching of scene solves.

A scene's final state is the same alone on the server, in a mix of other
scenes admitted while it runs, and on the plain single-scene per-step path
(bit for bit: the scenes share no device data and each runs its kernels in a
fixed order on its own stream). Admission respects the memory budget, and
results, release and errors follow the C ABI's contract.
"""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STEPS = 60


@pytest.fixture(scope="module")
def A():
    from sphgpu import _capi
    _capi.load()
    return _capi


def _scenes():
    from sphgpu import scenes
    return {
        "a": scenes.serving_dam_break(6000, "SESPH", stiffness=2000.0, viscosity=0.02, rest_density=900.0, seed=1),
        "b": scenes.serving_dam_break(20000, "IISPH", viscosity=0.005, rest_density=1200.0, seed=2),
        "c": scenes.serving_dam_break(9000, "SESPH", stiffness=4000.0, viscosity=0.001, rest_density=600.0, seed=3),
        "d": scenes.serving_dam_break(30000, "IISPH", viscosity=0.03, rest_density=700.0, seed=4),
    }


def _plain(A, sc, steps):
    from sphgpu import scenes
    g = scenes.build_system(sc)
    g.step_forward_in_time(steps)
    x, v = g.download(A.FIELD_POSITION), g.download(A.FIELD_VELOCITY)
    g.close()
    return x, v


def test_result_is_the_same_alone_in_a_mix_and_on_the_plain_path(A):
    from sphgpu.server import SceneServer
    sc = _scenes()
    with SceneServer(chunk_steps=20) as srv:
        alone = {}
        for key in ("a", "b"):
            t = srv.submit(sc[key], STEPS, keep_state=True)
            r = srv.wait(t, 300)
            assert r is not None and r["status"] == A.SPH_OK and r["steps"] == STEPS
            alone[key] = srv.fetch_state(t, r["particles"])
        # the mix: a and b arrive while c and d are already on the device
        tickets = {k: srv.submit(sc[k], STEPS, keep_state=True) for k in ("c", "d", "a", "b")}
        mixed = {}
        for k, t in tickets.items():
            r = srv.wait(t, 300)
            assert r is not None and r["status"] == A.SPH_OK
            mixed[k] = srv.fetch_state(t, r["particles"])
        st = srv.stats()
        assert st["completed"] == 6 and st["peak_active"] >= 2
    for key in ("a", "b"):
        x_p, v_p = _plain(A, sc[key], STEPS)
        for got in (alone[key], mixed[key]):
            assert np.array_equal(got[0], x_p)
            assert np.array_equal(got[1], v_p)


def test_admission_keeps_reserved_bytes_within_the_budget(A):
    from sphgpu import scenes
    from sphgpu.server import SceneServer
    sc = _scenes()["a"]
    with SceneServer() as probe:
        r = probe.wait(probe.submit(sc, 1), 120)
        est = r["device_bytes_reserved"]
    with SceneServer(memory_budget_bytes=int(1.5 * est), max_active=8, chunk_steps=10) as srv:
        ts = [srv.submit(sc, 20) for _ in range(4)]
        rs = [srv.wait(t, 300) for t in ts]
        assert all(r["status"] == A.SPH_OK for r in rs)
        st = srv.stats()
        assert st["peak_active"] == 1
        assert st["peak_reserved_bytes"] <= int(1.5 * est)
        # admitted in arrival order, one after the other
        for r0, r1 in zip(rs, rs[1:]):
            assert r1["start_s"] >= r0["finish_s"] - 1e-3
        big = scenes.serving_dam_break(60000, "SESPH")
        with pytest.raises(A.SPHError) as e:
            srv.submit(big, 10)
        assert e.value.code == A.SPH_ERR_CAPACITY


def test_poll_release_and_errors(A):
    from sphgpu import scenes
    from sphgpu.server import SceneServer
    with SceneServer() as srv:
        sc = scenes.serving_dam_break(40000, "SESPH")
        t = srv.submit(sc, 200)
        assert srv.poll(t) is None  # still being built or stepped
        r = srv.wait(t, 300)
        assert r["status"] == A.SPH_OK and r["steps"] == 200
        assert r["latency_s"] > 0 and r["finish_s"] >= r["start_s"] >= r["submit_s"]
        assert abs(r["time"] - 200 * 1e-3) < 1e-9
        with pytest.raises(A.SPHError) as e:
            srv.fetch_state(t, r["particles"])
        assert e.value.code == A.SPH_ERR_STATE
        srv.release(t)
        with pytest.raises(A.SPHError) as e:
            srv.poll(t)
        assert e.value.code == A.SPH_ERR_INVALID


def test_destroy_with_queued_and_running_scenes_returns(A):
    from sphgpu import scenes
    from sphgpu.server import SceneServer
    srv = SceneServer(max_active=1, chunk_steps=5)
    sc = scenes.serving_dam_break(30000, "IISPH")
    for _ in range(3):
        srv.submit(sc, 400)
    time.sleep(0.5)
    t0 = time.time()
    srv.close()
    assert time.time() - t0 < 60


def test_a_scene_that_fails_to_build_reports_its_error(A):
    """IISPHwOST only pairs with TakePredicted (sph/setup/mod.rs:229-231): the
    request is accepted, its build fails on the setup thread, and its result
    carries the error status while other scenes still complete."""
    from sphgpu import scenes
    from sphgpu.server import SceneServer
    bad = scenes.serving_dam_break(5000, "IISPH", seed=11)
    bad.procedures = dict(bad.procedures, pressure_solver="IISPHwOST")  # EulerCromer stays
    good = scenes.serving_dam_break(5000, "SESPH", seed=12)
    with SceneServer() as srv:
        tb, tg = srv.submit(bad, 10), srv.submit(good, 10)
        rb, rg = srv.wait(tb, 120), srv.wait(tg, 120)
    assert rb["status"] == A.SPH_ERR_INVALID and rb["steps"] == 0
    assert rg["status"] == A.SPH_OK and rg["steps"] == 10
