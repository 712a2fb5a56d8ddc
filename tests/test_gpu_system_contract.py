"""The SPHSystem contract of the reference's system-level tests
(simulation_lib/tests/sph/mod.rs:149-530) and of its system constructor's
(tests/sph/setup/mod.rs:286-465), restated on the engine through the C ABI:
a fluid-only scene (no boundary geometry) built the way the reference's
minimal scene is, stepped, measured, read back and cloned, for every solver
with its integration scheme, and the pairings the constructor refuses.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SPACING = 0.02
DT = 1e-3


@pytest.fixture(scope="module")
def A():
    from sphgpu import _capi
    _capi.load()
    return _capi


def _scene(cfl=False):
    from sphgpu import scenes
    pos = scenes.lattice_block((8, 8, 8), SPACING, origin=(0.0, 0.0, 0.0), jitter=0.01, seed=3)
    params = {"rest_density_grid_spacing": SPACING, "kernel_support_radius": 2 * SPACING,
              "disable_particles_below": -50.0, "fluid_viscosity": 0.01, "boundary_viscosity": 0.02,
              "boundary_pressure_acceleration_weighting": 0.7, "boundary_rest_volume_weighting": 1.0,
              "stiffness": 1000.0, "time_increment": DT}
    if cfl:
        params.update(max_time_increment=2e-3, cfl_number=0.4)
    return scenes.Scene(
        procedures={"kernel_function": "CubicBSpline3D", "integration_scheme": "EulerCromer",
                    "pressure_solver": "SESPH", "neighbor_search": "SpatialHashing",
                    "boundary_handling": "StaticSampleBoundary"},
        parameters=params, cfl_time_step=cfl, position=pos, mass=np.full(pos.shape[0], 1000.0 * SPACING ** 3))


def _system(cfl=False):
    from sphgpu import scenes
    return scenes.build_system(_scene(cfl))


def test_time_bookkeeping_of_fresh_and_stepped_systems(A):
    # mod.rs:149-214: a fresh system is at time 0 with no steps; every step
    # counts once; fixed steps advance time by exactly the increment and
    # CFL steps never move it backwards
    g = _system()
    assert g.time_steps_propagated() == 0 and abs(g.time()) < 1e-12
    g.step_forward_in_time()
    assert g.time_steps_propagated() == 1
    g.step_forward_in_time()
    assert g.time_steps_propagated() == 2
    g.step_forward_in_time()
    assert abs(g.time() - 3 * DT) < 1e-9
    g.close()
    c = _system(cfl=True)
    prev = c.time()
    for _ in range(3):
        c.step_forward_in_time()
        assert c.time() >= prev - 1e-12
        prev = c.time()
    assert c.time_steps_propagated() == 3
    c.close()


def test_measurement_reflects_the_configured_parameters(A):
    # mod.rs:217-253: SESPH passes its stiffness through verbatim and a fixed
    # step reports the configured increment
    g = _system()
    m = g.take_measurement()
    p = _scene().parameters
    for key in ("fluid_viscosity", "boundary_viscosity", "rest_density_grid_spacing", "kernel_support_radius",
                "stiffness"):
        assert m[key] == p[key], key
    assert m["time_step_size"] == DT
    g.close()


def test_fluid_readbacks_of_a_fresh_system(A):
    # mod.rs:256-270, 317-375: ids and positions of matching nonzero length,
    # every quantity one finite value per particle, a fluid sampled at rest
    # has zero speed and kinetic energy, and update() has already given every
    # particle a positive volume
    g = _system()
    ids, pos = g.get_fluid_ids(), g.get_fluid_pos()
    assert len(ids) > 0 and len(ids) == len(pos) and np.all(ids == 0)
    for q in (A.Q_SPEED, A.Q_VOLUME, A.Q_DENSITY, A.Q_DENSITY_ERROR, A.Q_PRESSURE, A.Q_KINETIC_ENERGY):
        v = g.get_quantity_of_fluid_samples(q)
        assert v.shape == (len(ids),) and np.all(np.isfinite(v)), q
    assert np.all(g.get_quantity_of_fluid_samples(A.Q_SPEED) == 0.0)
    assert np.all(g.get_quantity_of_fluid_samples(A.Q_KINETIC_ENERGY) == 0.0)
    assert np.all(g.get_quantity_of_fluid_samples(A.Q_VOLUME) > 0.0)
    # mod.rs:378-396: the quantity at a particle's own position
    vol = g.get_quantity_at_positions(A.Q_VOLUME, pos[:1])
    assert vol.shape == (1,) and np.isfinite(vol[0]) and vol[0] > 0
    speed = g.get_quantity_at_positions(A.Q_SPEED, pos[:1])
    assert speed.shape == (1,) and np.isfinite(speed[0])
    g.close()


def test_surface_boundary_views_and_checkpoint_without_boundary_geometry(A):
    # mod.rs:416-479: a surface for the fluid id present; with no boundary
    # geometry the boundary views are empty (Samples and TriangleMesh) and
    # the checkpoint holds no rigid states
    from sphgpu import formats as F
    g = _system()
    assert any(fid == 0 and len(idx) > 0 for fid, _, idx in g.reconstruct_surfaces())
    pos = g.get_fluid_pos()
    got = g.encode_time_step_info("samples", "uniform")
    want = F.encode_frame(g.time_steps_propagated(), g.take_measurement(), {"kind": "samples", "positions": pos},
                          {"positions": np.zeros((0, 3)), "coloring": "uniform"})
    assert got == want
    got = g.encode_time_step_info("samples", "uniform", boundary="triangle_mesh", boundary_coloring="original",
                                  render_meshes=[])
    want = F.encode_frame(g.time_steps_propagated(), g.take_measurement(), {"kind": "samples", "positions": pos},
                          {"kind": "triangle_mesh", "meshes": [], "poses": np.zeros((0, 7)),
                           "coloring": "original"})
    assert got == want
    assert g.get_checkpoint().boundaries == []
    g.close()


def test_checkpoint_restores_steps_state_and_time(A):
    # mod.rs:273-314, 482-504: a restored system continues from the saved
    # step count, fluid state and time; the RON text round-trips the state
    from sphgpu import formats as F
    a = _system()
    a.step_forward_in_time(2)
    ck = a.get_checkpoint()
    back = F.decode_checkpoint(F.encode_checkpoint(ck, A.FORMAT_RON), A.FORMAT_RON)
    assert back.time_steps_propagated == ck.time_steps_propagated
    assert np.array_equal(back.position, ck.position)
    b = _system()
    b.restore_checkpoint(back)
    assert b.time_steps_propagated() == 2
    assert abs(b.time() - a.time()) < 1e-9
    assert np.array_equal(b.get_fluid_ids(), a.get_fluid_ids())
    for f in (A.FIELD_POSITION, A.FIELD_VELOCITY, A.FIELD_MASS):
        assert np.array_equal(b.download(f), a.download(f)), f
    a.close()
    b.close()


def test_clones_evolve_independently(A):
    # mod.rs:507-529
    g = _system()
    c = g.clone()
    assert c.time_steps_propagated() == g.time_steps_propagated() == 0
    g.step_forward_in_time()
    assert g.time_steps_propagated() == 1 and c.time_steps_propagated() == 0
    g.close()
    c.close()


def test_every_pressure_solver_builds_and_steps_with_its_integrator(A):
    # setup/mod.rs:382-431: each solver with the scheme it pairs with, on
    # volume-map handling without geometry; a sweep cap bounds IISPH here
    from sphgpu import scenes
    for solver, scheme in (("SESPH", "EulerCromer"), ("SESPHwSplitting", "EulerCromer"), ("IISPH", "EulerCromer"),
                           ("IISPHwOST", "TakePredicted")):
        sc = _scene()
        sc.procedures = dict(sc.procedures, pressure_solver=solver, integration_scheme=scheme,
                             boundary_handling="VolumeMapBoundary")
        g = scenes.build_system(sc, extra_parameters={"max_solver_iterations": 100})
        t0 = g.time()
        g.step_forward_in_time()
        assert g.time() >= t0 and g.time_steps_propagated() == 1, solver
        assert np.all(np.isfinite(g.download(A.FIELD_POSITION))), solver
        g.close()


def test_pairing_checks_of_the_system_constructor(A):
    # setup/mod.rs:286-336 and the pairing rules of setup/mod.rs:229-244:
    # IISPHwOST only with TakePredicted and never with a dynamic boundary
    from sphgpu import scenes
    for solver, scheme in (("SESPH", "TakePredicted"), ("IISPHwOST", "EulerCromer")):
        sc = _scene()
        sc.procedures = dict(sc.procedures, pressure_solver=solver, integration_scheme=scheme)
        with pytest.raises(A.SPHError) as e:
            scenes.build_system(sc)
        assert e.value.code == A.SPH_ERR_INVALID
    sc = scenes.floating_cube_scene()
    sc.procedures = dict(sc.procedures, pressure_solver="IISPHwOST", integration_scheme="TakePredicted")
    with pytest.raises(A.SPHError) as e:
        scenes.build_system(sc)
    assert e.value.code == A.SPH_ERR_INVALID and "dynamic" in str(e.value)
