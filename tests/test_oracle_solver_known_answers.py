"""Pins the oracle's pressure solvers to the reference's solver unit tests,
restated against the oracle (paths under simulation_lib/):
  SESPH      tests/sph/pressure_solver/sesph.rs:309-633
  gravity, viscosity  src/sph/non_pressure_accelerations.rs:473-964
  IISPH      src/sph/pressure_solver/iisph.rs:714-1081
  SESPHwSplitting  src/sph/pressure_solver/sesph_with_splitting.rs:428-660
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


# ---- gravity and viscosity (non_pressure_accelerations.rs:473-964) ------------------
G = 9.81


def _np(oracle, pos, vel=None, **kw):
    pos = np.asarray(pos, np.float64).reshape(-1, 3)
    n = pos.shape[0]
    vel = np.zeros((n, 3)) if vel is None else vel
    return oracle.nonpressure_probe(H, SPACING, pos, vel, kw.pop("mass", np.full(n, 0.5)),
                                    kw.pop("vol", np.full(n, 0.02)), **kw)


def test_radial_gravity_pulls_toward_the_center(oracle):
    acc, _, _ = _np(oracle, [[2.0, 0, 0]], gravity=(0.0, 0.0, 0.0), viscosity=False)
    d = np.array([-2.0, 0.0, 0.0])
    assert np.linalg.norm(acc[0] - G * d / np.sqrt(d @ d + 1e-4)) < 1e-9


def test_radial_gravity_adds_onto_the_existing_acceleration(oracle):
    only, _, _ = _np(oracle, [[1.0, 0, 0]], gravity=(0.0, 0.0, 0.0), viscosity=False)
    both, _, _ = _np(oracle, [[1.0, 0, 0]], gravity=(0.0, 0.0, 0.0), viscosity=False, acc=[[3.0, -2.0, 1.0]])
    assert np.linalg.norm(both[0] - (np.array([3.0, -2.0, 1.0]) + only[0])) < 1e-9


def test_radial_gravity_is_finite_at_the_center(oracle):
    acc, _, _ = _np(oracle, [[0.0, 0, 0]], gravity=(0.0, 0.0, 0.0), viscosity=False)
    assert np.array_equal(acc[0], [0.0, 0.0, 0.0])


def test_radial_gravity_acts_on_each_particle(oracle):
    acc, _, _ = _np(oracle, [[1.0, 0, 0], [0, 2.0, 0]], gravity=(0.0, 0.0, 0.0), viscosity=False)
    assert acc[0, 0] < 0 and acc[1, 1] < 0


def test_radial_gravity_pulls_dynamic_bodies_and_skips_static_ones(oracle):
    _, f, _ = _np(oracle, [[50.0, 50, 50]], gravity=(0.0, 0.0, 0.0), viscosity=False,
                  boundary_pos=[[60.0, 60, 60]], boundary_vol=[0.01], body_com=[3.0, 0.0, 0.0])
    assert f[0] < 0 and abs(f[1]) < 1e-12 and abs(f[2]) < 1e-12
    _, f, _ = _np(oracle, [[50.0, 50, 50]], gravity=(0.0, 0.0, 0.0), viscosity=False,
                  boundary_pos=[[60.0, 60, 60]], boundary_vol=[0.01])
    assert not f.any()


def test_uniform_gravity_is_constant(oracle):
    acc, f, _ = _np(oracle, [[5.0, 0, 0], [-3.0, 7.0, 2.0]], gravity="uniform", viscosity=False,
                    boundary_pos=[[100.0, 0, 0]], boundary_vol=[0.01], body_com=[100.0, 0.0, 0.0])
    assert np.array_equal(acc[0], [0.0, 0.0, -G]) and np.array_equal(acc[1], [0.0, 0.0, -G])
    assert np.array_equal(f, [0.0, 0.0, -G])  # unit body mass


def _visc_term(oracle, nu, vol_j, xi, xj, vi, vj):
    r = np.asarray(xi) - np.asarray(xj)
    return nu * 2.0 * (3.0 + 2.0) * vol_j * (np.asarray(vi) - np.asarray(vj)) @ r / (
        r @ r + 0.01 * SPACING ** 2) * _grad(oracle, r)


def test_fluid_viscosity_matches_the_formula(oracle):
    pos = np.array([[0.0, 0, 0], [0.3, 0, 0], [0, 0.3, 0]])
    vel = np.eye(3)
    vol = np.array([0.02, 0.025, 0.03])
    acc, _, _ = _np(oracle, pos, vel, vol=vol, fluid_viscosity=5.0, boundary_viscosity=5.0)
    for i in range(3):
        want = sum(_visc_term(oracle, 5.0, vol[j], pos[i], pos[j], vel[i], vel[j]) for j in range(3))
        assert np.linalg.norm(acc[i] - want) < 1e-9


def test_fluid_viscosity_vanishes_for_equal_velocities(oracle):
    v = np.array([[2.0, -1.0, 0.5]] * 2)
    acc, _, _ = _np(oracle, [[0.0, 0, 0], [0.3, 0, 0]], v, fluid_viscosity=5.0, boundary_viscosity=5.0)
    assert np.abs(acc).max() < 1e-12


def test_fluid_viscosity_is_linear_in_the_viscosity(oracle):
    v = np.array([[1.0, 0, 0], [-1.0, 0, 0]])
    a1, _, _ = _np(oracle, [[0.0, 0, 0], [0.3, 0, 0]], v, fluid_viscosity=2.0, boundary_viscosity=2.0)
    a2, _, _ = _np(oracle, [[0.0, 0, 0], [0.3, 0, 0]], v, fluid_viscosity=4.0, boundary_viscosity=4.0)
    assert np.linalg.norm(a2[0] - 2.0 * a1[0]) < 1e-9


def test_viscosity_without_neighbors_is_zero(oracle):
    acc, _, _ = _np(oracle, [[0.0, 0, 0]], [[1.0, 0, 0]], fluid_viscosity=5.0, boundary_viscosity=5.0,
                    fluid_neighbors=False)
    assert np.array_equal(acc[0], [0.0, 0.0, 0.0])


def test_boundary_viscosity_static_and_dynamic(oracle):
    bpos = np.array([0.2, 0.0, 0.0])
    want = _visc_term(oracle, 5.0, 0.01, [0, 0, 0], bpos, [1.0, 0, 0], [0, 0, 0])
    acc, f, _ = _np(oracle, [[0.0, 0, 0]], [[1.0, 0, 0]], boundary_viscosity=5.0, fluid_neighbors=False,
                    boundary_pos=[bpos], boundary_vol=[0.01])
    assert np.linalg.norm(acc[0] - want) < 1e-9 and not f.any()
    acc, f, t = _np(oracle, [[0.0, 0, 0]], [[1.0, 0, 0]], boundary_viscosity=5.0, fluid_neighbors=False,
                    boundary_pos=[bpos], boundary_vol=[0.01], body_com=[5.0, 0.0, 0.0])
    assert np.linalg.norm(f - (-0.5 * acc[0])) < 1e-9
    assert np.linalg.norm(t - np.cross(bpos - np.array([5.0, 0, 0]), f)) < 1e-12


def test_boundary_viscosity_acts_per_particle(oracle):
    acc, f, _ = _np(oracle, [[0.0, 0, 0], [0.0, 1.0, 0]], [[1.0, 0, 0], [0, 1.0, 0]], boundary_viscosity=5.0,
                    fluid_neighbors=False, boundary_pos=[[0.2, 0, 0], [0.0, 1.2, 0]], boundary_vol=[0.01, 0.01],
                    body_com=[10.0, 0.0, 0.0])
    assert abs(acc[0, 0]) > 1e-12 and abs(acc[1, 1]) > 1e-12


# ---- IISPH source terms, diagonal, initialization (pressure_solver/iisph.rs:714-1081) ----
DT = 0.05


def test_iisph_vde_source_term_is_zero_without_neighbors(oracle):
    s_f, _ = oracle.iisph_terms_probe(H, SPACING, DT, 0.0, "vde", [[0, 0, 0]], [[1.0, 0, 0]], [0.5], [0.02],
                                      fluid_neighbors=False)
    assert s_f[0] == 0.0


def test_iisph_vde_source_term_matches_the_formula(oracle):
    pos = np.array([[0.0, 0, 0], [0.3, 0, 0]])
    vel = np.array([[1.0, 0, 0], [-1.0, 0, 0]])
    vol = np.array([0.02, 0.02])
    s_f, _ = oracle.iisph_terms_probe(H, SPACING, DT, 0.0, "vde", pos, vel, [0.5, 0.5], vol)
    want = -sum(DT * vol[j] * (vel[0] - vel[j]) @ _grad(oracle, pos[0] - pos[j]) for j in range(2))
    assert abs(s_f[0] - want) < 1e-9


def test_iisph_vp_source_term_keeps_the_volume_deviation(oracle):
    s_f, _ = oracle.iisph_terms_probe(H, SPACING, DT, 0.0, "vp", [[0, 0, 0]], [[0.0, 0, 0]], [0.5], [0.5 * RV],
                                      fluid_neighbors=False)
    assert abs(s_f[0] - (1.0 - RV / (0.5 * RV))) < 1e-9


def test_iisph_diagonal_is_zero_for_an_isolated_particle(oracle):
    _, a = oracle.iisph_terms_probe(H, SPACING, DT, 0.0, "diag", [[0, 0, 0]], [[0.0, 0, 0]], [0.5], [RV],
                                    fluid_neighbors=False)
    assert a[0] == 0.0


def test_iisph_diagonal_with_a_boundary_neighbor(oracle):
    w, bpos, bvol = 0.5, np.array([0.2, 0.0, 0.0]), 0.01
    _, a = oracle.iisph_terms_probe(H, SPACING, DT, w, "diag", [[0, 0, 0]], [[0.0, 0, 0]], [0.5], [RV],
                                    fluid_neighbors=False, boundary_pos=[bpos], boundary_vol=[bvol])
    sum_b = bvol * _grad(oracle, -bpos)
    c_f = -RV / 0.5 * (2.0 * w * sum_b)
    want = DT * DT * (c_f @ sum_b)
    assert abs(a[0] - want) < 1e-9 and a[0] <= 0.0


def test_iisph_initialize_cases(oracle):
    # near-zero diagonal -> 0; clamped negative -> 0; unclamped negative kept; positive formula
    assert oracle.iisph_initialize_probe([-5.0], [0.0], 0.5, 1e-6, True)[0] == 0.0
    assert oracle.iisph_initialize_probe([1.0], [-2.0], 0.5, 1e-9, True)[0] == 0.0
    p = oracle.iisph_initialize_probe([1.0], [-2.0], 0.5, 1e-9, False)[0]
    assert abs(p - 0.5 * 1.0 / -2.0) < 1e-9 and p < 0.0
    p = oracle.iisph_initialize_probe([-1.0], [-2.0], 0.5, 1e-9, True)[0]
    assert abs(p - 0.5 * -1.0 / -2.0) < 1e-9 and p > 0.0


# ---- SESPHwSplitting (pressure_solver/sesph_with_splitting.rs:428-660) ----------------
def test_splitting_predicted_density_of_an_isolated_particle_is_zero(oracle):
    rho, p, acc, _, _ = oracle.splitting_probe(H, SPACING, DT, 100.0, 0.0, [[0, 0, 0]], [[1.0, 0, 0]], [0.5],
                                               fluid_neighbors=False, acc=[[0.0, 0.0, -9.81]])
    # density_pred = 0 -> volume = inf -> max(V0 / inf - 1, 0) = 0
    assert rho[0] == 0.0 and p[0] == 0.0
    assert np.array_equal(acc[0], [0.0, 0.0, -9.81])


def test_splitting_predicted_density_with_fluid_neighbors(oracle):
    pos = np.array([[0.0, 0, 0], [0.3, 0, 0]])
    vel = np.array([[1.0, 0, 0], [-1.0, 0, 0]])
    mass = np.array([0.5, 0.6])
    rho, _, _, _, _ = oracle.splitting_probe(H, SPACING, DT, 100.0, 0.0, pos, vel, mass)
    want = sum(mass[j] * oracle.kernel_function(pos[0] - pos[j], H)
               + DT * (vel[0] - vel[j]) @ _grad(oracle, pos[0] - pos[j]) for j in range(2))
    assert abs(rho[0] - want) < 1e-9


def test_splitting_predicted_density_with_a_boundary_neighbor(oracle):
    bpos, bvol = np.array([0.2, 0.0, 0.0]), 0.01
    rho, _, _, _, _ = oracle.splitting_probe(H, SPACING, DT, 100.0, 0.0, [[0, 0, 0]], [[1.0, 0, 0]], [0.5],
                                             fluid_neighbors=False, boundary_pos=[bpos], boundary_vol=[bvol])
    want = bvol * (0.5 / RV) * oracle.kernel_function(-bpos, H) + DT * np.array([1.0, 0, 0]) @ _grad(oracle, -bpos)
    assert abs(rho[0] - want) < 1e-9


def test_splitting_pressures_of_a_compressed_pair(oracle):
    pos = np.array([[0.0, 0, 0], [0.3, 0, 0]])
    mass = np.array([0.5, 0.5])
    rho, p, _, _, _ = oracle.splitting_probe(H, SPACING, DT, 500.0, 0.0, pos, np.zeros((2, 3)), mass)
    for i in range(2):
        want_rho = sum(mass[j] * oracle.kernel_function(pos[i] - pos[j], H) for j in range(2))
        assert abs(p[i] - 500.0 * max(RV / (mass[i] / want_rho) - 1.0, 0.0)) < 1e-9


def test_splitting_reaction_on_a_dynamic_body(oracle):
    _, _, acc, f, _ = oracle.splitting_probe(H, SPACING, DT, 500.0, 1.0, [[0, 0, 0]], [[0.0, 0, 0]], [0.5],
                                             vol=[0.5 * RV], fluid_neighbors=False, boundary_pos=[[0.2, 0, 0]],
                                             boundary_vol=[0.01], body_com=[5.0, 0.0, 0.0])
    assert np.linalg.norm(f - (-0.5 * acc[0])) < 1e-9
