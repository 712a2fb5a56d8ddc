"""Pins the oracle's pressure solvers to the reference's solver unit tests,
restated against the oracle (paths under simulation_lib/):
  SESPH  tests/sph/pressure_solver/sesph.rs:309-633
The tests build the solver's inputs directly (positions, masses and volumes,
an empty or hashed fluid neighbor list, one boundary sample) and check the
pressures, the pressure accelerations and the reaction on a dynamic body.
"""
import numpy as np

H = 1.0
SPACING = 0.3
RV = SPACING * SPACING * SPACING  # SystemParameters' rest volume, spacing.powi(3) as products


def _grad(oracle, r):
    return np.asarray(oracle.kernel_gradient(r, H))


def test_sesph_pressure_is_zero_at_or_above_rest_volume(oracle):
    p, _, _, _ = oracle.sesph_probe(H, SPACING, 1000.0, 0.0, [[0, 0, 0], [1000, 0, 0]], [0.5, 0.5], [RV, 1.5 * RV])
    assert p[0] == 0.0 and p[1] == 0.0


def test_sesph_pressure_follows_the_state_equation(oracle):
    p, _, _, _ = oracle.sesph_probe(H, SPACING, 800.0, 0.0, [[0, 0, 0]], [0.5], [0.8 * RV])
    assert abs(p[0] - 800.0 * (RV / (0.8 * RV) - 1.0)) < 1e-9


def test_sesph_pressure_scales_linearly_with_stiffness(oracle):
    p1 = oracle.sesph_probe(H, SPACING, 100.0, 0.0, [[0, 0, 0]], [0.5], [0.5 * RV])[0][0]
    p2 = oracle.sesph_probe(H, SPACING, 200.0, 0.0, [[0, 0, 0]], [0.5], [0.5 * RV])[0][0]
    assert abs(p2 - 2.0 * p1) < 1e-9


def test_sesph_pressure_is_per_particle(oracle):
    vol = [0.9 * RV, 0.5 * RV]
    p, _, _, _ = oracle.sesph_probe(H, SPACING, 500.0, 0.0, [[0, 0, 0], [1000, 0, 0]], [0.5, 0.5], vol)
    for i in range(2):
        assert abs(p[i] - 500.0 * (RV / vol[i] - 1.0)) < 1e-9


def test_sesph_cluster_acceleration_matches_the_formula(oracle):
    pos = np.array([[0.0, 0.0, 0.0], [0.3, 0.0, 0.0], [0.0, 0.3, 0.0]])
    vol = np.array([0.9, 0.8, 0.7]) * RV
    mass = np.full(3, 0.5)
    p, acc, _, _ = oracle.sesph_probe(H, SPACING, 500.0, 0.0, pos, mass, vol)
    want_p = 500.0 * np.maximum(RV / vol - 1.0, 0.0)
    assert np.allclose(p, want_p, rtol=0, atol=1e-9)
    for i in range(3):
        want = np.zeros(3)
        for j in range(3):  # all three are neighbors (and i itself, whose gradient is zero)
            want -= vol[i] / mass[i] * vol[j] * (want_p[i] + want_p[j]) * _grad(oracle, pos[i] - pos[j])
        assert np.linalg.norm(acc[i] - want) < 1e-9


def test_sesph_adds_onto_the_existing_acceleration(oracle):
    _, acc, _, _ = oracle.sesph_probe(H, SPACING, 500.0, 0.0, [[0, 0, 0]], [0.5], [RV], acc=[[0.0, 0.0, -9.81]])
    assert np.array_equal(acc[0], [0.0, 0.0, -9.81])


def test_sesph_boundary_term_static_boundary_has_no_reaction(oracle):
    w, bpos, bvol = 0.5, np.array([0.2, 0.0, 0.0]), 0.01
    p, acc, f, t = oracle.sesph_probe(H, SPACING, 500.0, w, [[0, 0, 0]], [0.5], [0.5 * RV], fluid_neighbors=False,
                                      boundary_pos=[bpos], boundary_vol=[bvol])
    force = 2.0 * w * (0.5 * RV) * bvol * p[0] * _grad(oracle, -bpos)
    assert np.linalg.norm(acc[0] - (-force / 0.5)) < 1e-9
    assert not f.any() and not t.any()


def test_sesph_boundary_term_reacts_on_a_dynamic_body(oracle):
    bpos, com = np.array([0.2, 0.0, 0.0]), np.array([5.0, 0.0, 0.0])
    p, acc, f, t = oracle.sesph_probe(H, SPACING, 500.0, 1.0, [[0, 0, 0]], [0.5], [0.5 * RV], fluid_neighbors=False,
                                      boundary_pos=[bpos], boundary_vol=[0.01], body_com=com)
    force_on_fluid = 0.5 * acc[0]
    assert np.linalg.norm(f - (-force_on_fluid)) < 1e-9
    # applied at the sample: the torque about the center of mass
    assert np.linalg.norm(t - np.cross(bpos - com, f)) < 1e-12
