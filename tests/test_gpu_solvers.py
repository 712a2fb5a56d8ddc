"""GPU parity of the remaining solver/integrator/boundary variants (through
the C ABI, against the f64 oracle): SESPHwSplitting, IISPHwOST with
TakePredicted on two fluids, a dynamic StaticSampleBoundary body (two-way
RigidBodyMotion coupling), radial gravity; plus checkpoint restore, clone,
the host-buffer step and the GPU volume-map field builder.

f64 engine: 1e-9 relative of the oracle. f32 engine: bounds stated per test.
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


def _fields_close(g, o, A, oracle, precision, vol_tol=None, acc_tol=None):
    tol64 = 1e-9
    V_g, V_o = g.download(A.FIELD_VOLUME), o.download(oracle.F_VOLUME)
    assert rel_err(V_g, V_o, 1e-30) < (tol64 if precision == "f64" else (vol_tol or 1e-5))
    a_g, a_o = g.download(A.FIELD_ACCELERATION), o.download(oracle.F_ACCELERATION)
    sc = np.abs(a_o).max()
    assert np.max(np.abs(a_g - a_o)) <= (1e-7 if precision == "f64" else (acc_tol or 5e-3)) * sc


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_sesph_with_splitting_matches_oracle(A, oracle, precision):
    from sphgpu import scenes
    sc = scenes.dam_break_sesph_8k()
    sc.procedures = dict(sc.procedures, pressure_solver="SESPHwSplitting")
    g = scenes.build_system(sc, precision=precision)
    o = build_oracle(sc)
    _fields_close(g, o, A, oracle, precision)
    p_g, p_o = g.download(A.FIELD_PRESSURE), o.download(oracle.F_PRESSURE)
    assert np.max(np.abs(p_g - p_o)) <= (1e-8 if precision == "f64" else 2e-3) * np.abs(p_o).max()
    vs_g, vs_o = g.download(A.FIELD_PREDICTED_VELOCITY), o.download(oracle.F_SOLVER_VEL)
    assert np.max(np.abs(vs_g - vs_o)) < (1e-12 if precision == "f64" else 1e-5)
    g.step_forward_in_time(10)
    o.step(10)
    x_g, x_o = g.download(A.FIELD_POSITION), o.download(oracle.F_POSITION)
    assert np.max(np.abs(x_g - x_o)) < (1e-10 if precision == "f64" else 1e-6)


def _two_fluid_ost_scene():
    from sphgpu import scenes
    sc = scenes.dam_break_iisph_box(n_side=14, spacing=0.02, box=(0.6, 0.32, 0.32))
    sc.procedures = dict(sc.procedures, pressure_solver="IISPHwOST", integration_scheme="TakePredicted")
    sc.parameters = dict(sc.parameters, max_solver_iterations=30, fluid_viscosity=0.005,
                         boundary_viscosity=0.005)
    # split by a plane into rest densities 1000 and 500 (masses follow)
    pos = sc.position
    side = (pos @ np.array([0.3, 0.5, 0.8])) > np.median(pos @ np.array([0.3, 0.5, 0.8]))
    sc.fluid_id = side.astype(np.uint32)
    sc.mass = np.where(side, 500.0, 1000.0) * 0.02 ** 3
    return sc


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_iisph_w_ost_take_predicted_two_fluids(A, oracle, precision):
    from sphgpu import scenes
    sc = _two_fluid_ost_scene()
    verts, faces = sc.mesh
    fields = oracle.build_fields(verts, faces, 0.08, 0.04, 30)
    g = scenes.build_system(sc, precision=precision, fields=fields)
    o = build_oracle(sc, fields=fields)
    _fields_close(g, o, A, oracle, precision, acc_tol=5e-2)
    xi_g, xi_o = g.download(A.FIELD_INTEGRATOR_POSITION), o.download(oracle.F_INTEGRATOR_POS)
    vi_g, vi_o = g.download(A.FIELD_INTEGRATOR_VELOCITY), o.download(oracle.F_INTEGRATOR_VEL)
    assert np.max(np.abs(xi_g - xi_o)) < (1e-10 if precision == "f64" else 1e-5)
    assert np.max(np.abs(vi_g - vi_o)) < (1e-8 if precision == "f64" else 5e-3)
    mg, mo = g.take_measurement(), o.measurement()
    assert mg["solver_iterations"] == mo["solver_iterations"]
    if precision == "f64":
        assert abs(mg["predicted_density_error"] - mo["predicted_density_error"]) < 1e-8
    assert np.array_equal(g.get_fluid_ids(), sc.fluid_id)
    for _ in range(2):
        g.step_forward_in_time(1)
        o.step(1)
    x_g, x_o = g.download(A.FIELD_POSITION), o.download(oracle.F_POSITION)
    assert np.max(np.abs(x_g - x_o)) < (1e-9 if precision == "f64" else 1e-5)


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_dynamic_sample_boundary_two_way_coupling(A, oracle, precision):
    from sphgpu import scenes
    sc = scenes.floating_cube_scene()
    g = scenes.build_system(sc, precision=precision)
    o = build_oracle(sc)
    nb = sc.sample_boundaries[1][0].shape[0]
    assert rel_err(g.boundary_volumes(1, nb), o.boundary_volumes(1, nb), 1e-30) < (
        1e-9 if precision == "f64" else 1e-5)
    _fields_close(g, o, A, oracle, precision)
    # forces accumulated during the update (gravity + fluid reactions) pending
    # for the next step, then the body motion over a few steps
    st_g, st_o = g.rigid_state(1), o.rigid_state(1)
    assert np.allclose(st_g[13:19], st_o[13:19], rtol=1e-8 if precision == "f64" else 1e-3,
                       atol=1e-9 * np.abs(st_o[13:19]).max())
    for _ in range(5):
        g.step_forward_in_time(4)
        o.step(4)
    st_g, st_o = g.rigid_state(1), o.rigid_state(1)
    assert np.max(np.abs(st_g[0:3] - st_o[0:3])) < (1e-10 if precision == "f64" else 1e-6)  # com
    assert np.max(np.abs(st_g[3:7] - st_o[3:7])) < (1e-10 if precision == "f64" else 1e-6)  # orientation
    assert np.max(np.abs(st_g[7:10] - st_o[7:10])) < (1e-9 if precision == "f64" else 1e-4)  # velocity
    x_g, x_o = g.download(A.FIELD_POSITION), o.download(oracle.F_POSITION)
    assert np.max(np.abs(x_g - x_o)) < (1e-10 if precision == "f64" else 1e-5)


def test_radial_gravity_matches_oracle(A, oracle):
    from sphgpu import scenes
    from sphgpu.system import GpuSystem, make_config
    sc = scenes.dam_break_sesph_8k(n_side=10)
    center = (0.05, -0.1, 0.2)
    cfg = make_config(sc.procedures, sc.parameters, precision="f64", gravity={"type": "Radial", "center": center})
    g = GpuSystem(cfg)
    g.upload_fluid(sc.position, None, sc.mass)
    g.add_sample_boundary(sc.sample_boundaries[0][0])
    g.initialize()
    ocfg = dict(sc.parameters, integration_scheme=0, pressure_solver=0, boundary_handling=0, cfl_time_step=0,
                gravity_mode=1, gravity_center=center)
    o = oracle.OracleSystem(ocfg)
    o.upload_fluid(sc.position, None, sc.mass)
    o.add_sample_boundary(sc.sample_boundaries[0][0])
    o.initialize()
    a_g, a_o = g.download(A.FIELD_ACCELERATION), o.download(oracle.F_ACCELERATION)
    assert np.max(np.abs(a_g - a_o)) < 1e-8 * np.abs(a_o).max()


def test_checkpoint_restore_and_clone_reproduce_the_run(A):
    from sphgpu import scenes
    sc = scenes.dam_break_sesph_8k(n_side=12)
    a = scenes.build_system(sc, precision="f32")
    a.step_forward_in_time(10)
    ck = a.get_fluid_checkpoint()
    c = a.clone()
    a.step_forward_in_time(15)
    c.step_forward_in_time(15)
    b = scenes.build_system(sc, precision="f32")
    b.continue_from_checkpoint(ck)
    assert b.time_steps_propagated() == 10 and abs(b.time() - 0.01) < 1e-15
    b.step_forward_in_time(15)
    xa = a.download(A.FIELD_POSITION)
    assert np.array_equal(xa, c.download(A.FIELD_POSITION))
    assert np.array_equal(xa, b.download(A.FIELD_POSITION))
    assert a.time_steps_propagated() == c.time_steps_propagated() == b.time_steps_propagated() == 25


def test_host_buffer_step_equals_device_step(A):
    from sphgpu import scenes
    sc = scenes.dam_break_sesph_8k(n_side=12)
    a = scenes.build_system(sc, precision="f32")
    b = scenes.build_system(sc, precision="f32")
    a.step_forward_in_time(3)
    n = b.n
    xin, vin = b.download(A.FIELD_POSITION), b.download(A.FIELD_VELOCITY)
    xout, vout = np.zeros((n, 3)), np.zeros((n, 3))
    for _ in range(3):
        b.step_host(1, xin, vin, xout, vout)
        xin, vin = xout.copy(), vout.copy()
    assert np.array_equal(a.download(A.FIELD_POSITION), xout)
    assert np.array_equal(a.download(A.FIELD_VELOCITY), vout)


def test_host_buffer_step_readback_cases(A):
    """sph_step_host reads the last step's state back while that step's
    update still runs: several steps in one call, an IISPH scene, and a step
    that disables particles (renumbered afterwards, read back at the end)
    all return what the device path downloads."""
    from sphgpu import scenes
    for sc, steps in ((scenes.dam_break_sesph_8k(n_side=12), 3),
                      (scenes.serving_dam_break(2000, solver="IISPH"), 2)):
        a = scenes.build_system(sc, precision="f32")
        b = scenes.build_system(sc, precision="f32")
        n = b.n
        xin, vin = b.download(A.FIELD_POSITION), b.download(A.FIELD_VELOCITY)
        xout, vout = np.zeros((n, 3)), np.zeros((n, 3))
        a.step_forward_in_time(steps)
        b.step_host(steps, xin, vin, xout, vout)
        assert np.array_equal(a.download(A.FIELD_POSITION), xout)
        assert np.array_equal(a.download(A.FIELD_VELOCITY), vout)
    sc = scenes.dam_break_sesph_8k(n_side=12)
    sc.parameters = dict(sc.parameters, disable_particles_below=-0.29)
    a = scenes.build_system(sc, precision="f32")
    b = scenes.build_system(sc, precision="f32")
    n = b.n
    xin, vin = b.download(A.FIELD_POSITION), b.download(A.FIELD_VELOCITY)
    xin[::50, 2] = -0.295  # below the threshold: disabled by the step's update
    a.step_host(1, xin, vin, None, None)
    xout, vout = np.zeros((n, 3)), np.zeros((n, 3))
    b.step_host(1, xin, vin, xout, vout)
    assert a.n == b.n < n
    assert np.array_equal(a.download(A.FIELD_POSITION), xout[:b.n])
    assert np.array_equal(a.download(A.FIELD_VELOCITY), vout[:b.n])


@pytest.mark.parametrize("mesh", ["box", "sphere"])
def test_gpu_volume_map_field_builder_matches_oracle(oracle, mesh):
    from sphgpu import scenes
    from sphgpu.fields import build_volume_map_fields
    if mesh == "box":
        verts = scenes.transform_mesh(scenes.CUBE_VERTICES, scale=(0.32, 0.16, 0.16))
        faces = scenes.CUBE_FACES_INWARD
    else:
        verts, faces = scenes.icosphere(2, radius=0.3, inward=True)
    dx, r = 0.08, 0.04
    sdf_g, vm_g = build_volume_map_fields(verts, faces, dx, r, 30)
    sdf_o, vm_o = oracle.build_fields(verts, faces, dx, r, 30)
    for a, b in ((sdf_g, sdf_o), (vm_g, vm_o)):
        assert np.array_equal(a.n, b.n) and np.allclose(a.x_min, b.x_min) and np.allclose(a.x_max, b.x_max)
        assert np.array_equal(np.isnan(a.nodes), np.isnan(b.nodes))
        m = ~np.isnan(b.nodes)
        assert m.sum() > 0
        assert np.max(np.abs(a.nodes[m] - b.nodes[m])) <= 1e-12 * max(1.0, np.abs(b.nodes[m]).max())
