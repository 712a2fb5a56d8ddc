"""Reduced-scale cases of two benchmark configurations.

* IISPHwOST two-fluid ball in a sphere container (the precision study): the
  f64 engine follows the f64 oracle; the f32 engine's per-field error
  against the f64 engine after 20 steps is reported and bounded.
* IISPH tank with eight two-way coupled rigid bodies (4 cubes, 4 spheres),
  all StaticSampleBoundary, CFL steps: body states and fluid positions
  follow the oracle.
"""
import numpy as np
import pytest

from conftest import build_oracle, rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def A():
    from sphgpu import _capi
    _capi.load()
    return _capi


@pytest.fixture(scope="module")
def ball():
    from sphgpu import scenes
    from sphgpu.fields import build_volume_map_fields
    sc = scenes.two_fluid_ball(radius=0.25, spacing=0.02, seed=3, subdivisions=3)
    sc.parameters = dict(sc.parameters, max_solver_iterations=30)
    verts, faces = sc.mesh
    return sc, build_volume_map_fields(verts, faces, 0.08, 0.04)


def test_two_fluid_ball_f64_engine_follows_oracle(A, oracle, ball):
    from sphgpu import scenes
    sc, fields = ball
    g = scenes.build_system(sc, precision="f64", fields=fields)
    o = build_oracle(sc, fields=fields)
    assert rel_err(g.download(A.FIELD_VOLUME), o.download(oracle.F_VOLUME), 1e-30) < 1e-9
    for _ in range(2):
        g.step_forward_in_time(5)
        o.step(5)
    assert np.max(np.abs(g.download(A.FIELD_POSITION) - o.download(oracle.F_POSITION))) < 1e-10
    assert g.take_measurement()["solver_iterations"] == o.measurement()["solver_iterations"]


def test_two_fluid_ball_f32_error_against_f64(A, ball):
    from sphgpu import scenes
    sc, fields = ball
    out = {}
    for prec in ("f64", "f32"):
        g = scenes.build_system(sc, precision=prec, fields=fields)
        g.step_forward_in_time(20)
        out[prec] = {f: g.download(f) for f in (A.FIELD_POSITION, A.FIELD_VELOCITY, A.FIELD_VOLUME,
                                                A.FIELD_PRESSURE)}
        g.close()
    ref, got = out["f64"], out["f32"]
    h = sc.parameters["rest_density_grid_spacing"]
    err = {
        "position_max_over_spacing": np.max(np.abs(got[A.FIELD_POSITION] - ref[A.FIELD_POSITION])) / h,
        "velocity_max_rel": np.max(np.abs(got[A.FIELD_VELOCITY] - ref[A.FIELD_VELOCITY]))
        / np.abs(ref[A.FIELD_VELOCITY]).max(),
        "volume_max_rel": rel_err(got[A.FIELD_VOLUME], ref[A.FIELD_VOLUME], 1e-30),
        "pressure_max_rel_to_max": np.max(np.abs(got[A.FIELD_PRESSURE] - ref[A.FIELD_PRESSURE]))
        / max(np.abs(ref[A.FIELD_PRESSURE]).max(), 1.0),
    }
    print("f32 vs f64 after 20 steps:", {k: float(f"{v:.3e}") for k, v in err.items()})
    assert err["position_max_over_spacing"] < 1e-3
    assert err["velocity_max_rel"] < 2e-2
    assert err["volume_max_rel"] < 1e-3
    assert err["pressure_max_rel_to_max"] < 1e-1


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_rigid_body_tank_follows_oracle(A, oracle, precision):
    from sphgpu import scenes
    sc = scenes.rigid_body_tank(seed=2)
    g = scenes.build_system(sc, precision=precision)
    o = build_oracle(sc)
    for _ in range(3):
        g.step_forward_in_time(3)
        o.step(3)
    assert abs(g.time() - o.time()) < (1e-12 if precision == "f64" else 1e-6)
    for b in range(1, len(sc.sample_boundaries)):
        st_g, st_o = g.rigid_state(b), o.rigid_state(b)
        assert np.max(np.abs(st_g[0:3] - st_o[0:3])) < (1e-10 if precision == "f64" else 1e-6), b
        assert np.max(np.abs(st_g[3:7] - st_o[3:7])) < (1e-10 if precision == "f64" else 1e-5), b
        assert np.max(np.abs(st_g[7:10] - st_o[7:10])) < (1e-9 if precision == "f64" else 1e-4), b
    x_g, x_o = g.download(A.FIELD_POSITION), o.download(oracle.F_POSITION)
    assert np.max(np.abs(x_g - x_o)) < (1e-10 if precision == "f64" else 1e-5)
