"""Quantities at arbitrary positions (sph_get_quantity_at_positions) against
the oracle's restatement of SPHSystem::get_quantity_at_positions
(sph/mod.rs:241-341, sums of sph/quantities.rs:14-330).

Evaluation points are sensor planes through the fluid, the walls and the
bodies, plus points on particles, between them and far outside. Each case
covers all six ScalarQuantity values: speed and volume with sample
boundaries (static and a rotating body) and with volume maps (static and a
rotating body), and the fluid-only sums. The f64 engine is held to 1e-6 of
the oracle (the sums run in f64 in both, in different orders, and are cast
to f32); the f32 engine to 1e-4, the size of its state's rounding (for
volumes: of their kernel sums), except for pressures: near rest they are
small differences of densities, and the IISPH solve in f32 stops within the
target density error, so they are held to 2e-2 of the largest pressure.
"""
import numpy as np
import pytest

from conftest import build_oracle

pytestmark = pytest.mark.gpu

QUANTITIES = range(6)
QUANTITY_VOLUME = 1
QUANTITY_PRESSURE = 4


@pytest.fixture(scope="module")
def A():
    from sphgpu import _capi
    _capi.load()
    return _capi


def _plane(lo, hi, axis, at, n):
    """n x n points spanning [lo, hi] in the two axes other than `axis`."""
    a, b = [d for d in range(3) if d != axis]
    u = np.linspace(lo[a], hi[a], n)
    v = np.linspace(lo[b], hi[b], n)
    U, V = np.meshgrid(u, v, indexing="ij")
    P = np.empty((n * n, 3))
    P[:, a], P[:, b], P[:, axis] = U.ravel(), V.ravel(), at
    return P


def _eval_points(sc, n=48, seed=0):
    pos = sc.position
    lo, hi = pos.min(0) - 0.1, pos.max(0) + 0.1
    mid = 0.5 * (pos.min(0) + pos.max(0))
    rng = np.random.default_rng(seed)
    pts = [_plane(lo, hi, 1, mid[1], n), _plane(lo, hi, 2, mid[2], n),
           pos[rng.choice(len(pos), 200, replace=False)],
           rng.uniform(lo, hi, size=(300, 3)),
           np.array([[50.0, 50.0, 50.0], [-3.0, 0.0, 0.0]])]
    return np.concatenate(pts).astype(np.float32)


def _compare(got, want, rtol):
    got = np.asarray(got, np.float64)
    want = np.asarray(want, np.float64)
    inf = np.isinf(want)
    assert np.array_equal(np.isinf(got), inf)
    assert np.all(got[inf] == want[inf])
    g, w = got[~inf], want[~inf]
    floor = max(np.abs(w).max(), 1e-30) * rtol
    err = np.abs(g - w) / np.maximum(np.abs(w), floor)
    assert err.max() < rtol, (err.max(), int(err.argmax()))


def _compare_volume_sums(got, want, V0, atol):
    """Volumes through their kernel sums sum V0 W / V0 (about 1 inside the
    fluid, 0 where the volume is infinite). An f32 state moves positions by
    an ulp, which changes W of a neighbor at the support's edge by a large
    factor but by little in absolute terms: where such a neighbor is a
    point's only one, the volume's relative error is large while its sum's
    absolute error stays at the rounding level."""
    sg = V0 / np.asarray(got, np.float64)
    sw = V0 / np.asarray(want, np.float64)
    err = np.abs(sg - sw)
    assert err.max() < atol, (err.max(), int(err.argmax()))


def _check_all(g, o, pts, rtol, quantities=QUANTITIES, precision="f64", spacing=None):
    for q in quantities:
        got, want = g.get_quantity_at_positions(q, pts), o.quantity_at_positions(q, pts)
        if q == QUANTITY_VOLUME and precision == "f32":
            _compare_volume_sums(got, want, spacing ** 3, rtol)
        elif q == QUANTITY_PRESSURE and precision == "f32":
            # near rest, SESPH pressures are k (rho / rho0 - 1) with rho / rho0 - 1
            # of a few 1e-3, so the f32 state's density rounding (~1e-5) moves
            # them by ~1e-2 of their largest value
            _compare(got, want, 2e-2)
        else:
            _compare(got, want, rtol)


def _with_velocity(sc, seed=1, scale=0.5):
    rng = np.random.default_rng(seed)
    sc.velocity = rng.normal(0.0, scale, size=sc.position.shape)
    return sc


@pytest.mark.parametrize("precision,rtol", [("f64", 1e-6), ("f32", 1e-4)])
def test_sample_boundary_scene_at_initialization(A, oracle, precision, rtol):
    from sphgpu import scenes
    sc = _with_velocity(scenes.dam_break_sesph_8k(n_side=12))
    g = scenes.build_system(sc, precision=precision)
    o = build_oracle(sc)
    pts = _eval_points(sc)
    # a plane through the container's wall samples as well
    pts = np.concatenate([pts, _plane((-0.32,) * 3, (0.32,) * 3, 0, -0.295, 40).astype(np.float32)])
    _check_all(g, o, pts, rtol, precision=precision, spacing=0.02)
    g.close()


def test_sesph_state_after_steps(A, oracle):
    """After 40 steps the oracle is rebuilt from the engine's state (its first
    update recomputes the same volumes and SESPH pressures)."""
    from sphgpu import scenes
    sc = scenes.dam_break_sesph_8k(n_side=12)
    g = scenes.build_system(sc, precision="f64")
    g.step_forward_in_time(40)
    sc.position = g.download(A.FIELD_POSITION)
    sc.velocity = g.download(A.FIELD_VELOCITY)
    sc.mass = g.download(A.FIELD_MASS)
    o = build_oracle(sc)
    _check_all(g, o, _eval_points(sc, seed=3), 1e-6)
    g.close()


@pytest.mark.parametrize("precision,rtol", [("f64", 1e-6), ("f32", 1e-4)])
def test_rotating_sample_body(A, oracle, precision, rtol):
    from sphgpu import scenes
    sc = _with_velocity(scenes.floating_cube_scene(), seed=2)
    g = scenes.build_system(sc, precision=precision)
    o = build_oracle(sc)
    body = sc.sample_boundaries[1][1]
    c = np.asarray(body.center_of_mass)
    pts = np.concatenate([_eval_points(sc, n=32),
                          _plane(c - 0.1, c + 0.1, 0, c[0], 40),
                          _plane(c - 0.1, c + 0.1, 2, c[2] - 0.05, 40)]).astype(np.float32)
    _check_all(g, o, pts, rtol, precision=precision, spacing=0.02)
    # the body's samples move: speed near it includes their velocities
    near = _plane(c - 0.07, c + 0.07, 0, c[0], 20).astype(np.float32)
    assert g.get_quantity_at_positions(A.Q_SPEED, near).max() > 0
    g.close()


def _vm_scene():
    from sphgpu import scenes
    from sphgpu.fields import build_volume_map_fields
    from sphgpu.system import RigidInit
    sc = _with_velocity(scenes.dam_break_iisph_box(n_side=12, spacing=0.02, box=(0.6, 0.32, 0.32)), seed=4)
    sc.parameters = dict(sc.parameters, max_solver_iterations=60)
    verts, faces = sc.mesh
    container = build_volume_map_fields(verts, faces, 0.08, 0.04)
    bv, bf = scenes.icosphere(2, 0.06)
    ball = build_volume_map_fields(bv, bf, 0.08, 0.04)
    mass = 600.0 * 4.0 / 3.0 * np.pi * 0.06 ** 3
    rigid = RigidInit(mass=mass, inertia_body=np.eye(3) * 0.4 * mass * 0.06 ** 2,
                      center_of_mass=(0.15, 0.0, 0.0), orientation=(np.cos(0.2), 0.0, np.sin(0.2), 0.0),
                      linear_velocity=(0.1, 0.0, -0.2), angular_velocity=(0.0, 0.0, 2.0))
    sc.volume_maps = [(container[0], container[1], None), (ball[0], ball[1], rigid)]
    return sc


@pytest.mark.parametrize("precision,rtol", [("f64", 1e-6), ("f32", 1e-4)])
def test_volume_maps_static_and_rotating(A, oracle, precision, rtol):
    from sphgpu import scenes
    sc = _vm_scene()
    g = scenes.build_system(sc, precision=precision)
    o = build_oracle(sc)
    c = np.array([0.15, 0.0, 0.0])
    pts = np.concatenate([_eval_points(sc, n=32),
                          _plane((-0.3, -0.16, -0.16), (0.3, 0.16, 0.16), 1, 0.0, 48),
                          _plane(c - 0.09, c + 0.09, 2, 0.01, 40)]).astype(np.float32)
    _check_all(g, o, pts, rtol, quantities=[q for q in QUANTITIES if q != A.Q_PRESSURE],
               precision=precision, spacing=0.02)
    # IISPH pressures: the f32 Jacobi solve stops within the target density
    # error of the f64 one, not at its rounding
    _compare(g.get_quantity_at_positions(A.Q_PRESSURE, pts), o.quantity_at_positions(A.Q_PRESSURE, pts),
             rtol if precision == "f64" else 2e-2)
    near = _plane(c - 0.08, c + 0.08, 2, 0.0, 24).astype(np.float32)
    assert g.get_quantity_at_positions(A.Q_SPEED, near).max() > 0
    g.close()


def test_errors_empty_input_and_unchanged_state(A):
    from sphgpu import scenes
    from sphgpu.system import GpuSystem, make_config
    sc = scenes.dam_break_sesph_8k(n_side=10)
    g = scenes.build_system(sc)
    pts = _eval_points(sc, n=16)
    for q in (-1, 6):
        with pytest.raises(A.SPHError) as e:
            g.get_quantity_at_positions(q, pts)
        assert e.value.code == A.SPH_ERR_INVALID
    assert g.get_quantity_at_positions(A.Q_VOLUME, np.zeros((0, 3))).shape == (0,)
    far = g.get_quantity_at_positions(A.Q_VOLUME, [[40.0, 40.0, 40.0]])
    assert np.isposinf(far[0])
    # evaluating changes nothing the next steps use
    g.step_forward_in_time(10)
    for q in QUANTITIES:
        g.get_quantity_at_positions(q, pts)
    g.step_forward_in_time(10)
    ref = scenes.build_system(sc)
    ref.step_forward_in_time(20)
    assert np.array_equal(g.download(A.FIELD_POSITION), ref.download(A.FIELD_POSITION))
    assert np.array_equal(g.download(A.FIELD_VELOCITY), ref.download(A.FIELD_VELOCITY))
    g.close()
    ref.close()
    # before initialize
    params = dict(sc.parameters, device=0)
    s = GpuSystem(make_config(sc.procedures, params, precision="f32", cfl_time_step=False))
    s.upload_fluid(sc.position, None, sc.mass, None)
    with pytest.raises(A.SPHError) as e:
        s.get_quantity_at_positions(A.Q_SPEED, pts)
    assert e.value.code == A.SPH_ERR_STATE
    s.close()
