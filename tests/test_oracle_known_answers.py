"""Pins the oracle to the reference's own known-answer tests.

The reference (Rust) cannot be built here, so the oracle's fidelity rests on
the formula-level assertions of the reference's test suite, restated below
against the oracle (sim_lib = simulation_lib):
  kernel      tests/sph/kernel/cubic_spline.rs:17-232
  hashing     src/neighbor_search/spatial_hashing.rs:173-390,
              tests/neighbor_search/spatial_hashing.rs:19-330
  volume      src/sph/quantities.rs:437-633
  quantities  src/sph/quantities.rs:437-800 through sph/mod.rs:241-341
  IISPH       tests/sph/pressure_solver/iisph.rs:429-490
  IISPHwOST   src/sph/pressure_solver/iisph_optimized_source_term.rs:530-582
  EulerCromer tests/sph/integration_schemes/euler_cromer.rs:91-300
  rigid body  tests/sph/boundary_handling/rigid_body_motion.rs:44-642
  serendipity tests/utilities/discretization.rs:21-212
  mesh SDF    src/sph/boundary_handling/volume_map_boundary.rs:2809-2835
"""
import math

import numpy as np
import pytest

from conftest import build_oracle

ALPHA = 16.0 / math.pi


# ---- kernel -------------------------------------------------------------------------
def test_kernel_known_values(oracle):
    assert abs(oracle.kernel_w(0.0) - 0.5) < 1e-12
    assert abs(oracle.kernel_w(0.5) - 0.125) < 1e-12
    for q in (1.0, 1.5, 10.0):
        assert oracle.kernel_w(q) == 0.0
    assert oracle.kernel_dqw(1.0) == 0.0 and oracle.kernel_dqw(2.0) == 0.0
    h = 1.0
    assert oracle.kernel_function([1.0, 0, 0], h) == 0.0
    assert abs(oracle.kernel_function([0, 0, 0], 2.0) - ALPHA / 8.0 * 0.5) < 1e-12


def test_kernel_derivative_matches_finite_difference(oracle):
    eps = 1e-6
    for q in (0.05, 0.2, 0.35, 0.55, 0.7, 0.9):
        num = (oracle.kernel_w(q + eps) - oracle.kernel_w(q - eps)) / (2 * eps)
        assert abs(oracle.kernel_dqw(q) - num) < 1e-4


def test_kernel_gradient_zero_at_origin_and_antisymmetric(oracle):
    assert np.all(oracle.kernel_gradient([0, 0, 0], 1.0) == 0.0)
    r = np.array([0.1, -0.2, 0.3])
    g1, g2 = oracle.kernel_gradient(r, 1.0), oracle.kernel_gradient(-r, 1.0)
    assert np.allclose(g1, -g2, atol=1e-15)
    # gradient points from the neighbor towards the evaluated point: W decreases
    assert np.dot(g1, r) < 0


def test_kernel_trait_default_methods(oracle):
    """KernelFn's default q / kernel_function / kernel_gradient
    (ST/sph/kernel/mod.rs:42-166, there on a dummy kernel, here on the cubic
    spline): W = alpha/h^3 w(|r|/h), grad W = alpha/h^4 r/|r| w'(q), radial
    symmetry, h^-3 and h^-4 scaling, a gradient parallel to r."""
    r, h = np.array([0.3, 0.4, 0.0]), 1.25  # |r| = 0.5, q = 0.4
    q = 0.5 / h
    assert abs(oracle.kernel_function(r, h) - ALPHA / h ** 3 * oracle.kernel_w(q)) < 1e-12
    g = oracle.kernel_gradient(r, h)
    assert np.linalg.norm(g - ALPHA / h ** 4 * r / 0.5 * oracle.kernel_dqw(q)) < 1e-12
    assert abs(oracle.kernel_function([0.5, 0, 0], h) - oracle.kernel_function([0, 0, -0.5], h)) < 1e-12
    a = np.array([0.2, -0.1, 0.3])
    for k in (2.0, 3.0):
        assert abs(oracle.kernel_function(k * a, k * h) - oracle.kernel_function(a, h) / k ** 3) < 1e-9
        assert np.linalg.norm(oracle.kernel_gradient(k * a, k * h) - oracle.kernel_gradient(a, h) / k ** 4) < 1e-9
    assert np.linalg.norm(np.cross(oracle.kernel_gradient(a, 1.0), a)) < 1e-12


def test_kernel_integrates_to_one(oracle):
    # radial Gauss-Legendre quadrature of 4 pi r^2 W(r) on the two polynomial
    # pieces [0, h/2] and [h/2, h] (exact for these degrees)
    x, w = oracle.gauss_legendre(8)
    h = 0.7
    tot = 0.0
    for a, b in ((0.0, 0.5 * h), (0.5 * h, h)):
        for xi, wi in zip(x, w):
            r = 0.5 * (b - a) * xi + 0.5 * (a + b)
            tot += 0.5 * (b - a) * wi * 4 * math.pi * r * r * oracle.kernel_function([r, 0, 0], h)
    assert abs(tot - 1.0) < 1e-12


# ---- spatial hashing ------------------------------------------------------------------
def test_map_int_to_uint_and_hash(oracle):
    assert [oracle.map_int_to_uint(k) for k in (0, 1, 5)] == [0, 2, 10]
    assert [oracle.map_int_to_uint(k) for k in (-1, -5)] == [3, 11]
    vals = [oracle.map_int_to_uint(k) for k in range(-100, 101)]
    assert len(set(vals)) == len(vals)
    assert oracle.cell_hash(0, 0, 0) != oracle.cell_hash(1, 0, 0)
    assert oracle.cell_hash(1, 2, 3) == oracle.cell_hash(1, 2, 3)
    # (2k)*73856093 ^ ... by hand
    assert oracle.cell_hash(1, -1, 2) == (2 * 73856093) ^ (3 * 19349663) ^ (4 * 83492791)


def test_hash_has_no_collisions_over_41_cubed(oracle):
    seen = set()
    for k in range(-20, 21):
        for l in range(-20, 21):
            for m in range(-20, 21):
                seen.add(oracle.cell_hash(k, l, m))
    assert len(seen) == 41 ** 3


@pytest.mark.parametrize("p,cs,cell", [
    ((0.5, 0.5, 0.5), 1.0, (0, 0, 0)), ((2.3, 4.7, 1.1), 1.0, (2, 4, 1)),
    ((-0.5, -1.5, -3.9), 1.0, (-1, -2, -4)), ((1.5, 3.0, 0.9), 2.0, (0, 1, 0)),
    ((1.0, 2.0, 3.0), 1.0, (1, 2, 3))])
def test_get_cell(oracle, p, cs, cell):
    assert tuple(oracle.get_cell(p, cs)) == cell


def _row(off, idx, i):
    return list(idx[int(off[i]):int(off[i + 1])])


def test_find_samples_semantics(oracle):
    # close neighbor + self
    off, idx, _ = oracle.find_samples(1.0, [[0, 0, 0], [0.5, 0, 0]], [[0, 0, 0], [0.5, 0, 0]])
    assert set(_row(off, idx, 0)) == {0, 1}
    # far neighbor excluded
    off, idx, _ = oracle.find_samples(2.0, [[0, 0, 0]], [[0, 0, 0], [10, 0, 0]], cell_size=1.0)
    assert _row(off, idx, 0) == [0]
    # exactly at the range: strict <
    off, idx, _ = oracle.find_samples(2.0, [[0, 0, 0]], [[0, 0, 0], [2, 0, 0]], cell_size=2.0)
    assert 1 not in _row(off, idx, 0)
    # negative positions and across zero
    off, idx, _ = oracle.find_samples(1.0, [[-1, -1, -1]], [[-1, -1, -1], [-1.5, -1, -1]])
    assert 1 in _row(off, idx, 0)
    off, idx, _ = oracle.find_samples(0.2, [[-0.05, 0, 0]], [[-0.05, 0, 0], [0.05, 0, 0]], cell_size=1.0)
    assert 1 in _row(off, idx, 0)


def test_find_samples_matches_brute_force(oracle):
    rng = np.random.default_rng(3)
    pts = rng.uniform(-1, 1, size=(600, 3))
    off, idx, dups = oracle.find_samples(0.25, pts, pts)
    assert dups == 0
    d = np.sqrt(((pts[:, None, :] - pts[None, :, :]) ** 2).sum(-1))
    for i in range(0, 600, 37):
        assert sorted(_row(off, idx, i)) == sorted(np.nonzero(d[i] < 0.25)[0].tolist())


# ---- volume / density -------------------------------------------------------------------
def _lattice(n, dx):
    g = np.arange(n) * dx
    return np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)


def _isolated_system(oracle, pos, vel=None, solver=0, integrator=0, dt=0.01, h=0.04, spacing=0.02,
                     mass=None):
    from sphgpu import scenes
    sc = scenes.Scene(
        procedures={"integration_scheme": "TakePredicted" if integrator else "EulerCromer",
                    "pressure_solver": ["SESPH", "SESPHwSplitting", "IISPH", "IISPHwOST"][solver],
                    "boundary_handling": "VolumeMapBoundary"},
        parameters={"rest_density_grid_spacing": spacing, "kernel_support_radius": h,
                    "disable_particles_below": -50.0, "fluid_viscosity": 0.0,
                    "boundary_viscosity": 0.0, "boundary_pressure_acceleration_weighting": 0.7,
                    "boundary_rest_volume_weighting": 1.0, "stiffness": 1000.0,
                    "target_density_error": 0.01, "relaxation_factor": 0.5,
                    "min_diagonal_element": 1e-9, "time_increment": dt},
        cfl_time_step=False, position=np.asarray(pos, np.float64),
        mass=np.full(len(pos), 1000.0 * spacing ** 3 if mass is None else mass),
        velocity=None if vel is None else np.asarray(vel, np.float64))
    return build_oracle(sc)


def test_volume_is_rest_volume_over_kernel_sum(oracle):
    h, dx = 0.04, 0.02
    pos = _lattice(7, dx)
    s = _isolated_system(oracle, pos, h=h, spacing=dx)
    V = s.download(oracle.F_VOLUME)
    V0 = dx ** 3
    i = 3 * 49 + 3 * 7 + 3  # lattice center
    acc = sum(V0 * oracle.kernel_function(pos[i] - pos[j], h) for j in range(len(pos))
              if np.linalg.norm(pos[i] - pos[j]) < h)
    assert abs(V[i] - V0 / acc) < 1e-12 * V0
    # the lattice interior recovers the rest density within 15 %
    rho = 1000.0 * dx ** 3 / V[i]
    assert abs(rho - 1000.0) / 1000.0 < 0.15


def test_isolated_particle_volume_is_inverse_self_weight(oracle):
    s = _isolated_system(oracle, [[0.1, 0.2, 0.3]])
    V = s.download(oracle.F_VOLUME)[0]
    assert abs(V - 1.0 / oracle.kernel_function([0, 0, 0], 0.04)) < 1e-15


# ---- integration --------------------------------------------------------------------------
def test_euler_cromer_recurrence_isolated_particle(oracle):
    # isolated SESPH particle: V > V0 so no pressure; acceleration = gravity
    x0, v0, dt = np.array([1.0, 2.0, 3.0]), np.array([0.5, -0.25, 0.125]), 0.01
    s = _isolated_system(oracle, [x0], [v0], dt=dt)
    g = np.array([0, 0, -9.81])
    assert np.allclose(s.download(oracle.F_ACCELERATION)[0], g, atol=1e-14)
    s.step(1)
    v1 = v0 + dt * g
    x1 = x0 + dt * v1  # position update uses the new velocity
    assert np.allclose(s.download(oracle.F_VELOCITY)[0], v1, atol=1e-12)
    assert np.allclose(s.download(oracle.F_POSITION)[0], x1, atol=1e-12)
    s.step(1)
    v2 = v1 + dt * g
    assert np.allclose(s.download(oracle.F_POSITION)[0], x1 + dt * v2, atol=1e-12)
    assert abs(s.time() - 2 * dt) < 1e-15


def test_iisph_w_ost_isolated_particle_trace(oracle):
    # iisph_optimized_source_term.rs:530-582: gravity only enters v*, the
    # acceleration is overwritten by the (zero) pressure acceleration.
    x0, v0, dt = np.array([1.0, 2.0, 3.0]), np.array([0.5, 0.0, 0.0]), 0.05
    s = _isolated_system(oracle, [x0], [v0], solver=3, integrator=1, dt=dt, h=1.0, spacing=0.3)
    g = np.array([0, 0, -9.81])
    assert s.download(oracle.F_PRESSURE)[0] == 0.0
    assert np.all(s.download(oracle.F_ACCELERATION)[0] == 0.0)
    v_pred = v0 + dt * g
    assert np.allclose(s.download(oracle.F_INTEGRATOR_VEL)[0], v_pred, atol=1e-9)
    assert np.allclose(s.download(oracle.F_INTEGRATOR_POS)[0], x0 + dt * v_pred, atol=1e-9)


# ---- IISPH ----------------------------------------------------------------------------------
def _probe_inputs():
    h, dt, spacing, gamma = 1.0, 0.05, 0.3, 0.5
    V = spacing ** 3 * 0.5   # compressed -> s_f < 0
    return dict(pos=[0, 0, 0], vel=[0, 0, 0], mass=0.5, volume=V, dt=dt, h=h, spacing=spacing,
                gamma_p=gamma, omega=0.5, eps=1e-9, bpos=[0.2, 0, 0], bvol=0.01)


def test_iisph_diagonal_and_initial_pressure_match_formula(oracle):
    a = _probe_inputs()
    p, aff, sf, it = oracle.iisph_probe(**a, after=-1)
    gb = a["bvol"] * oracle.kernel_gradient(-np.array(a["bpos"]), a["h"])
    c_f = -a["volume"] / a["mass"] * (2.0 * a["gamma_p"] * gb)
    aff_expected = a["dt"] ** 2 * np.dot(c_f, gb)
    s_expected = 1.0 - a["spacing"] ** 3 / a["volume"]
    assert abs(aff - aff_expected) < 1e-12 and aff < 0
    assert abs(sf - s_expected) < 1e-12
    # initialize(): p0 = max(omega s / a_ff, 0) (the value the reference test
    # asserts for its `AfterIteration(0)` call)
    p_expected = max(0.5 * s_expected / aff_expected, 0.0)
    assert abs(p - p_expected) < 1e-12 * p_expected and p > 0


def test_iisph_after_iteration_counts_follow_the_code(oracle):
    # converged(AfterIteration(n)) stops when iter > n: n+1 sweeps. One sweep
    # on an isolated particle with one boundary sample gives
    # p1 = (1 - omega) p0 + omega s / a_ff = 0.75 s / a_ff.
    a = _probe_inputs()
    p, aff, sf, it = oracle.iisph_probe(**a, after=0)
    assert it == 1
    assert abs(p - 0.75 * sf / aff) < 1e-12 * abs(0.75 * sf / aff)
    _, _, _, it3 = oracle.iisph_probe(**a, after=3)
    assert it3 == 4


def test_iisph_expansion_never_gives_negative_pressure(oracle):
    a = _probe_inputs()
    a["volume"] = a["spacing"] ** 3 * 2.0  # expanded -> s_f > 0
    p, aff, sf, _ = oracle.iisph_probe(**a, after=0)
    assert sf > 0 and p == 0.0


def test_iisph_isolated_particle_at_rest_volume_is_a_noop(oracle):
    """ST/sph/pressure_solver/iisph.rs:495-535: no neighbors -> zero diagonal,
    zero pressure, the pre-existing acceleration untouched. The test there
    expects 2 sweeps; the code's TargetDensityError stop (`iter > 2 && err <
    tde`, iisph.rs:378-393) gives 3, and the oracle follows the code."""
    acc0 = np.array([0.0, 0.0, -9.81])
    v0 = 0.3 * 0.3 * 0.3  # powi(3) multiplies, as the oracle's rest volume does
    p, acc, sweeps, err, _, _ = oracle.iisph_solve_probe(
        [0, 0, 0], [0, 0, 0], 0.5, v0, acc0, 0.05, 1.0, 0.3, 0.0, 0.5, 1e-9, 0.01)
    assert p == 0.0 and np.array_equal(acc, acc0)
    assert sweeps == 3 and err == 0.0


def test_iisph_registers_the_reaction_on_a_dynamic_body_once(oracle):
    """ST/sph/pressure_solver/iisph.rs:538-592: only the final pressure
    acceleration registers a reaction force, equal and opposite to the
    particle's pressure force, however many sweeps ran."""
    p, acc, sweeps, _, F, T = oracle.iisph_solve_probe(
        [0, 0, 0], [0, 0, 0], 0.5, 0.3 * 0.3 * 0.3 * 0.5, [0, 0, 0], 0.05, 1.0, 0.3, 1.0, 0.5, 1e-9, 0.01,
        bpos=[0.2, 0, 0], bvol=0.01, com=[5.0, 0, 0])
    assert p > 0 and sweeps >= 3 and np.linalg.norm(F) > 0
    assert np.linalg.norm(F - (-0.5 * acc)) < 1e-9
    assert np.linalg.norm(T - np.cross(np.array([0.2, 0, 0]) - [5.0, 0, 0], F)) < 1e-9


# ---- rigid body -----------------------------------------------------------------------------
def _rigid_init(mass=2.0, I=(1.0, 2.0, 3.0), com=(0, 0, 0), q=(1, 0, 0, 0), v=(0, 0, 0), w=(0, 0, 0)):
    Ib = np.diag(I)
    return np.concatenate([[mass], Ib.ravel(), np.linalg.inv(Ib).ravel(), com, q, v, w]).astype(np.float64)


def test_rigid_body_semi_implicit_linear_step(oracle):
    init = _rigid_init(mass=2.0)
    dt = 0.1
    st = oracle.rigid_body_step(init, [[0, 0, 4.0]], [[0, 0, 0]], dt, 1)
    v = 4.0 / 2.0 * dt
    assert np.allclose(st[7:10], [0, 0, v])
    assert np.allclose(st[0:3], [0, 0, v * dt])  # com uses the new velocity
    assert np.allclose(st[13:19], 0.0)           # forces reset after the step


def test_rigid_body_rotation_angle_is_preserved(oracle):
    # constant angular velocity about z for n steps -> rotation angle w n dt
    w, dt, n = 0.7, 0.01, 50
    init = _rigid_init(I=(1.0, 1.0, 1.0), w=(0, 0, w))
    st = oracle.rigid_body_step(init, [[0, 0, 0]], [[0, 0, 0]], dt, n)
    q = st[3:7]
    angle = 2 * math.atan2(np.linalg.norm(q[1:]), q[0])
    assert abs(angle - w * n * dt) < 1e-12
    assert abs(np.linalg.norm(q) - 1.0) < 1e-12


def test_rigid_body_torque_from_off_center_force(oracle):
    init = _rigid_init()
    st = oracle.rigid_body_step(init, [[0, 1.0, 0]], [[1.0, 0, 0]], 0.1, 1)
    # torque = r x F = (1,0,0) x (0,1,0) = (0,0,1); L = T dt
    assert np.allclose(st[10:13], [0, 0, 0.1])


# ---- serendipity / volume map --------------------------------------------------------------
def _field(oracle, fn, n=(2, 2, 2), dx=0.5, x_min=(0, 0, 0)):
    n = np.array(n)
    NX, NY, NZ = 3 * n + 1
    nodes = np.full(NX * NY * NZ, np.nan)
    for kz in range(NZ):
        for ky in range(NY):
            for kx in range(NX):
                # only nodes with at most one off-corner coordinate belong to a cell
                if sum(k % 3 != 0 for k in (kx, ky, kz)) <= 1:
                    p = np.array(x_min) + np.array([kx, ky, kz]) / 3.0 * dx
                    nodes[(kz * NY + ky) * NX + kx] = fn(p)
    x_min = np.array(x_min, np.float64)
    return oracle.Field(x_min, x_min + n * dx, dx, n, nodes)


def test_serendipity_reproduces_constant_and_linear_fields(oracle):
    F = _field(oracle, lambda p: 2.5)
    for p in ([0.1, 0.2, 0.3], [0.9, 0.7, 0.4], [0.5, 0.5, 0.5]):
        assert abs(F.function(p) - 2.5) < 1e-12
        assert np.allclose(F.gradient(p), 0.0, atol=1e-9)
    L = _field(oracle, lambda p: 1.0 + 2 * p[0] - p[1] + 0.5 * p[2])
    for p in ([0.1, 0.2, 0.3], [0.6, 0.35, 0.8]):
        assert abs(L.function(p) - (1.0 + 2 * p[0] - p[1] + 0.5 * p[2])) < 1e-9
        assert np.allclose(L.gradient(p), [2, -1, 0.5], atol=1e-6)
    assert F.function([2.0, 0.1, 0.1]) is None   # out of bounds


def test_serendipity_bounds_clamping_and_pruning(oracle):
    """ST/utilities/discretization.rs:116-190: out of bounds below and above
    the domain, the upper corner valid through clamping to the last cell, an
    entirely pruned domain (absent nodes) and a never-pruned one."""
    F = _field(oracle, lambda p: 0.0, n=(1, 1, 1), dx=1.0)
    assert F.function([-0.01, 0.5, 0.5]) is None and F.function([1.01, 0.5, 0.5]) is None
    C = _field(oracle, lambda p: 4.2, n=(1, 1, 1), dx=1.0)
    assert abs(C.function([1.0, 1.0, 1.0]) - 4.2) < 1e-9
    P = _field(oracle, lambda p: 0.0, n=(1, 1, 1), dx=1.0)
    P.nodes[:] = np.nan
    assert P.function([0.5, 0.5, 0.5]) is None
    N = _field(oracle, lambda p: -1000.0, n=(1, 1, 1), dx=1.0)
    assert abs(N.function([0.5, 0.5, 0.5]) + 1000.0) < 1e-6


def test_serendipity_gradient_interior_and_near_the_boundary(oracle):
    """ST/utilities/discretization.rs:192-230: central differences with
    h = dx/6 recover a linear field's gradient inside, and a stencil point
    beyond the domain is an error, not a one-sided fallback."""
    L = _field(oracle, lambda p: 2 * p[0] - p[1] + 0.5 * p[2], n=(2, 2, 2), dx=1.0, x_min=(-1, -1, -1))
    assert np.linalg.norm(L.gradient([0.0, 0.0, 0.0]) - [2, -1, 0.5]) < 1e-2
    one = _field(oracle, lambda p: 0.0, n=(1, 1, 1), dx=2.0, x_min=(-1, -1, -1))
    assert one.gradient([0.9, 0.0, 0.0]) is None


def test_gauss_legendre_ball_volume(oracle):
    # SDF uniformly far inside the boundary -> integrand 1 -> ball volume, and
    # the band case integrates the cubic extension function
    sdf = _field(oracle, lambda p: -0.01, n=(4, 4, 4), dx=0.5)
    r = 0.2
    assert abs(oracle.volume_at(sdf, [1.0, 1.0, 1.0], r) - 4 / 3 * math.pi * r ** 3) < 1e-12
    sdf0 = _field(oracle, lambda p: 0.0, n=(4, 4, 4), dx=0.5)
    v = oracle.volume_at(sdf0, [1.0, 1.0, 1.0], r)
    assert abs(v - 4 / 3 * math.pi * r ** 3) < 1e-9  # sd = 0 -> extension 1
    far = _field(oracle, lambda p: 5.0, n=(4, 4, 4), dx=0.5)
    assert oracle.volume_at(far, [1.0, 1.0, 1.0], r) == 0.0


def test_mesh_signed_distance_cube(oracle):
    from sphgpu import scenes
    out = scenes.CUBE_FACES_OUTWARD
    inw = scenes.CUBE_FACES_INWARD
    v = scenes.CUBE_VERTICES
    # outward cube: outside positive (face distance), inside negative
    assert abs(oracle.mesh_signed_distance(v, out, [2.5, 0.1, -0.2]) - 1.5) < 1e-12
    assert abs(oracle.mesh_signed_distance(v, out, [0.5, 0.1, -0.2]) + 0.5) < 1e-12
    # inward cube (a container): inside positive
    assert abs(oracle.mesh_signed_distance(v, inw, [0.5, 0.1, -0.2]) - 0.5) < 1e-12
    # outside near an edge: euclidean distance to the edge, negative for the container
    d = oracle.mesh_signed_distance(v, inw, [1.3, 1.4, 0.0])
    assert abs(d + math.hypot(0.3, 0.4)) < 1e-12


# ---- quantities at arbitrary positions (sensor planes) ------------------------------------
Q_SPEED, Q_VOLUME, Q_DENSITY, Q_DENSITY_ERROR, Q_PRESSURE, Q_KINETIC_ENERGY = range(6)


def _manual(oracle, s, eval_pts, h, term):
    """Sum of term(j) * W(x - x_j) over the fluid samples within h of each
    evaluation point (f64, the point taken as f32 like the reference)."""
    pos = s.download(oracle.F_POSITION)
    out = []
    for x in np.asarray(eval_pts, np.float32).astype(np.float64):
        acc = 0.0
        for j in range(len(pos)):
            if np.linalg.norm(x - pos[j]) < h:
                acc += term(j) * oracle.kernel_function(x - pos[j], h)
        out.append(acc)
    return np.array(out)


def test_quantity_volume_matches_formula_at_and_between_samples(oracle):
    # quantities.rs:437-535: V0 / sum V0 W, at the samples and at a point between them
    h, dx = 1.0, 0.3
    pos = [[0.0, 0.0, 0.0], [0.3, 0.0, 0.0], [0.0, 0.3, 0.0]]
    s = _isolated_system(oracle, pos, h=h, spacing=dx)
    ev = pos + [[0.15, 0.0, 0.0]]
    got = s.quantity_at_positions(Q_VOLUME, ev)
    V0 = dx ** 3
    want = V0 / _manual(oracle, s, ev, h, lambda j: V0)
    assert np.array_equal(got, want.astype(np.float32))


def test_quantity_volume_of_an_isolated_point_is_infinite(oracle):
    # quantities.rs:476-504: zero neighbor sum -> +inf
    s = _isolated_system(oracle, [[1000.0, 1000.0, 1000.0]], h=0.1, spacing=0.05)
    v = s.quantity_at_positions(Q_VOLUME, [[0.0, 0.0, 0.0]])
    assert np.isinf(v[0]) and v[0] > 0
    for q in (Q_SPEED, Q_DENSITY, Q_DENSITY_ERROR, Q_PRESSURE, Q_KINETIC_ENERGY):
        assert s.quantity_at_positions(q, [[0.0, 0.0, 0.0]])[0] == 0.0


def test_quantity_on_empty_input(oracle):
    # quantities.rs:542-561
    s = _isolated_system(oracle, [[0.0, 0.0, 0.0]])
    for q in range(6):
        assert s.quantity_at_positions(q, np.zeros((0, 3))).shape == (0,)
    with pytest.raises(ValueError):
        s.quantity_at_positions(6, [[0.0, 0.0, 0.0]])


def test_quantity_lattice_recovers_rest_density_and_volume(oracle):
    # quantities.rs:564-633: a lattice at rest spacing, h / dx = 4, evaluated at its center
    h, dx = 0.2, 0.05
    k = int(round(h / dx))
    g = np.arange(-k, k + 1) * dx
    pos = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    s = _isolated_system(oracle, pos, h=h, spacing=dx, mass=1000.0 * dx ** 3)
    rho = s.quantity_at_positions(Q_DENSITY, [[0.0, 0.0, 0.0]])[0]
    vol = s.quantity_at_positions(Q_VOLUME, [[0.0, 0.0, 0.0]])[0]
    assert abs(rho - 1000.0) / 1000.0 < 0.15
    assert abs(vol - dx ** 3) / dx ** 3 < 0.15


def test_quantity_speed_pressure_kinetic_energy_match_formulas(oracle):
    # quantities.rs:637-800, with the system's own volumes, velocities, masses and pressures
    h, dx = 1.0, 0.3
    pos = [[0.0, 0.0, 0.0], [0.4, 0.0, 0.0], [0.0, 0.4, 0.0]]
    vel = [[1.0, 0.0, 0.0], [0.0, 2.0, 0.0], [0.0, 0.0, 3.0]]
    s = _isolated_system(oracle, pos, vel=vel, h=h, spacing=dx, mass=[0.5, 0.6, 0.7])
    V = s.download(oracle.F_VOLUME)
    v = s.download(oracle.F_VELOCITY)
    m = s.download(oracle.F_MASS)
    p = s.download(oracle.F_PRESSURE)
    ev = pos + [[0.1, 0.2, 0.05], [0.9, 0.9, 0.9]]
    x = np.asarray(ev, np.float32).astype(np.float64)
    P = s.download(oracle.F_POSITION)
    sv = np.zeros((len(ev), 3))
    for i in range(len(ev)):
        for j in range(3):
            if np.linalg.norm(x[i] - P[j]) < h:
                sv[i] += v[j] * V[j] * oracle.kernel_function(x[i] - P[j], h)
    speed = s.quantity_at_positions(Q_SPEED, ev)
    assert np.allclose(speed, np.linalg.norm(sv, axis=1), rtol=1e-6, atol=0)
    pres = s.quantity_at_positions(Q_PRESSURE, ev)
    assert np.allclose(pres, _manual(oracle, s, ev, h, lambda j: p[j] * V[j]), rtol=1e-6, atol=1e-12)
    ke = s.quantity_at_positions(Q_KINETIC_ENERGY, ev)
    want = _manual(oracle, s, ev, h, lambda j: 0.5 * m[j] * (v[j] @ v[j]) * V[j])
    assert np.allclose(ke, want, rtol=1e-6, atol=0)
    rho = s.quantity_at_positions(Q_DENSITY, ev)
    assert np.allclose(rho, _manual(oracle, s, ev, h, lambda j: m[j]), rtol=1e-6, atol=0)


def test_quantity_density_error_takes_masses_in_the_volume_slot(oracle):
    # quantities.rs:682-718 with sph/mod.rs:302-311, which passes the fluid
    # MASSES as `sample_volumes`: neighbors whose mass is at or above the rest
    # volume are skipped, the others add (V0 / m - 1) m W
    h, dx = 1.0, 0.3
    V0 = dx ** 3
    pos = [[0.0, 0.0, 0.0], [0.2, 0.0, 0.0], [0.0, 0.2, 0.0]]
    masses = [V0, 1.5 * V0, 0.5 * V0]
    s = _isolated_system(oracle, pos, h=h, spacing=dx, mass=masses)
    got = s.quantity_at_positions(Q_DENSITY_ERROR, pos)
    want = 100.0 * _manual(oracle, s, pos, h, lambda j: (V0 / masses[j] - 1.0) * masses[j]
                           if masses[j] < V0 else 0.0)
    assert np.allclose(got, want, rtol=1e-6, atol=0)
    assert got[0] > 0
    # water-like masses (rest density 1000) are never below the rest volume: zero everywhere
    s2 = _isolated_system(oracle, pos, h=h, spacing=dx)
    assert np.all(s2.quantity_at_positions(Q_DENSITY_ERROR, pos) == 0.0)


# ---- SpatialHashing::find_samples (tests/neighbor_search/spatial_hashing.rs:19-330) --------
def _nb(oracle, rng_, pos, samples=None, cell=1.0):
    off, idx, _ = oracle.find_samples(rng_, pos, pos if samples is None else samples, cell_size=cell)
    return [sorted(_row(off, idx, i)) for i in range(len(pos))]


def test_hashing_empty_and_self(oracle):
    assert _nb(oracle, 2.0, np.zeros((0, 3))) == []
    assert _nb(oracle, 2.0, [[0, 0, 0]]) == [[0]]
    assert _nb(oracle, 2.0, [[0, 0, 0]], samples=np.zeros((0, 3))) == [[]]


def test_hashing_close_far_and_boundary_samples(oracle):
    assert _nb(oracle, 2.0, [[0, 0, 0], [0.5, 0, 0]]) == [[0, 1], [0, 1]]
    assert _nb(oracle, 2.0, [[0, 0, 0], [100, 0, 0]]) == [[0], [1]]
    assert _nb(oracle, 2.0, [[0, 0, 0]], samples=[[0.5, 0, 0], [100, 0, 0]]) == [[0]]


def test_hashing_is_symmetric_and_finds_clusters(oracle):
    nb = _nb(oracle, 1.5, [[0, 0, 0], [1, 0, 0], [0, 1, 0]])
    assert all(i in nb[j] for i in range(3) for j in nb[i])
    assert _nb(oracle, 1.0, [[0, 0, 0], [0.3, 0, 0], [0, 0.3, 0], [0, 0, 0.3]]) == [[0, 1, 2, 3]] * 4
    nb = _nb(oracle, 2.0, [[0, 0, 0], [0.5, 0, 0], [50, 50, 50], [50.5, 50, 50]])
    assert nb == [[0, 1], [0, 1], [2, 3], [2, 3]]


def test_hashing_range_diagonal_duplicates_and_cell_boundaries(oracle):
    assert 1 not in _nb(oracle, 1.0, [[0, 0, 0], [1.5, 0, 0]])[0]
    assert 1 in _nb(oracle, 2.0, [[0, 0, 0], [1.5, 0, 0]])[0]
    assert _nb(oracle, 1.0, [[0, 0, 0], [0.5, 0.5, 0.5]]) == [[0, 1], [0, 1]]
    assert _nb(oracle, 0.5, [[1, 1, 1], [1, 1, 1]]) == [[0, 1], [0, 1]]
    assert _nb(oracle, 1.0, [[0.9, 0, 0], [1.1, 0, 0]]) == [[0, 1], [0, 1]]


def test_hashing_repeated_calls_grow_and_shrink(oracle):
    assert 1 not in _nb(oracle, 2.0, [[0, 0, 0], [100, 0, 0]])[0]
    nb = _nb(oracle, 1.0, [[0, 0, 0], [0.5, 0, 0], [0.3, 0, 0], [100, 0, 0]])
    assert 2 in nb[0] and nb[3] == [3]
    assert _nb(oracle, 1.0, [[0, 0, 0], [0.5, 0, 0]]) == [[0, 1], [0, 1]]


def test_hashing_cell_size_is_only_a_performance_parameter(oracle):
    assert 1 not in _nb(oracle, 2.0, [[0, 0, 0], [5, 0, 0]], cell=10.0)[0]
    assert 1 in _nb(oracle, 6.0, [[0, 0, 0], [5, 0, 0]], cell=10.0)[0]
    # a cell size far below the range searches ceil(range / cell) cells each way
    assert _nb(oracle, 1.0, [[0, 0, 0], [0.5, 0, 0]], cell=0.1) == [[0, 1], [0, 1]]


def test_tiny_cube_volume_map_fields_give_usable_boundary_samples(oracle):
    """volume_map_boundary.rs:169-222 (ignored upstream for its runtime): a
    cube of half-size 0.1 with h = 0.045 and dx = 4 * 0.0225 builds fields
    in which a fluid particle on the cube's surface finds a boundary sample
    of positive, finite volume."""
    from sphgpu import scenes
    h, spacing = 0.045, 0.0225
    verts = scenes.CUBE_VERTICES * 0.1
    sdf, vm = oracle.build_fields(verts, scenes.CUBE_FACES_OUTWARD, 4 * spacing, h)
    sc = scenes.Scene(
        procedures={"integration_scheme": "EulerCromer", "pressure_solver": "SESPH",
                    "boundary_handling": "VolumeMapBoundary"},
        parameters={"rest_density_grid_spacing": spacing, "kernel_support_radius": h,
                    "disable_particles_below": -50.0, "time_increment": 1e-3},
        cfl_time_step=False, position=np.array([[0.1, 0.0, 0.0]]), mass=np.array([1000.0 * spacing ** 3]))
    s = build_oracle(sc, fields=(sdf, vm))
    has, xb, _, vol = s.vm_samples(0)
    assert has[0] and vol[0] > 0 and np.isfinite(vol[0])
