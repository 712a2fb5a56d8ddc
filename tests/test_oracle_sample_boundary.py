"""Pins the oracle's StaticSampleBoundary to the reference's unit tests
(simulation_lib/tests/sph/boundary_handling/static_sample_boundary.rs:116-600),
restated with the same cube, spacing, support radius and tolerances.

The reference samples its cube with sample_triangle_mesh_surface; here the
samples come from the host's restatement of that sampler
(sphgpu.scenes.sample_triangle_mesh_surface), and a dynamic cube of density
1000 gets the mass and inertia of a solid cube, as the mesh's mass properties
give it. The visualization and checkpoint tests of the same file are restated
against the engine's frame and checkpoint encoders elsewhere.
"""
import numpy as np
import pytest

SPACING = 0.5
KERNEL_SUPPORT_RADIUS = 1.2
WEIGHTING = 1.0


@pytest.fixture(scope="module")
def cube():
    from sphgpu import scenes
    return scenes.sample_triangle_mesh_surface(scenes.CUBE_VERTICES, scenes.CUBE_FACES_OUTWARD, SPACING)


def _rigid(translation=(0, 0, 0), velocity=(0, 0, 0), angular_velocity=(0, 0, 0)):
    from sphgpu import scenes
    mass = 1000.0 * 8.0
    I = scenes.box_inertia(mass, 2.0)
    return np.concatenate([[mass], I.ravel(), np.linalg.inv(I).ravel(), translation, [1, 0, 0, 0],
                           velocity, angular_velocity]).astype(np.float64)


def _static(oracle, cube):
    b = oracle.SampleBoundaries()
    b.add(cube)
    return b


def _dynamic(oracle, cube, *args):
    b = oracle.SampleBoundaries()
    b.add(cube, _rigid(*args))
    return b


# ---- construction ---------------------------------------------------------------------------
def test_new_sample_boundary_is_empty(oracle):
    assert len(oracle.SampleBoundaries()) == 0


def test_add_static_boundary_populates_and_is_not_dynamic(oracle, cube):
    b = _static(oracle, cube)
    assert len(b) == 1
    pos, _, _, com = b.samples(0)
    assert len(pos) == len(cube) and com is None


def test_add_dynamic_boundary_is_dynamic_with_center_of_mass_near_translation(oracle, cube):
    b = _dynamic(oracle, cube, (5, 0, 0))
    assert len(b) == 1
    com = b.samples(0)[3]
    assert com is not None and np.linalg.norm(com - [5, 0, 0]) < 1e-6


def test_dynamic_boundary_sample_positions_start_as_origin_placeholders_before_initialize(oracle, cube):
    assert np.array_equal(_dynamic(oracle, cube, (5, 0, 0)).samples(0)[0][0], [0, 0, 0])


# ---- samples on the cube surface ------------------------------------------------------------
def test_static_boundary_samples_lie_on_cube_surface(oracle, cube):
    m = np.abs(_static(oracle, cube).samples(0)[0]).max(axis=1)
    assert np.all(m <= 1.0 + 1e-9) and np.all(m >= 1.0 - 1e-9)


def test_dynamic_boundary_samples_are_offset_by_translation(oracle, cube):
    b = _dynamic(oracle, cube, (10, 0, 0))
    b.initialize(KERNEL_SUPPORT_RADIUS, WEIGHTING)
    x = b.samples(0)[0][:, 0]
    assert np.all(x >= 10 - 1 - 1e-6) and np.all(x <= 10 + 1 + 1e-6)


def test_initialize_moves_dynamic_boundary_samples_into_world_space(oracle, cube):
    b = _dynamic(oracle, cube, (5, 0, 0))
    b.initialize(KERNEL_SUPPORT_RADIUS, WEIGHTING)
    assert np.linalg.norm(b.samples(0)[0][0]) > 3.0


def test_initialize_assigns_positive_finite_volume_to_every_sample(oracle, cube):
    b = _static(oracle, cube)
    b.initialize(KERNEL_SUPPORT_RADIUS, WEIGHTING)
    vol = b.samples(0)[2]
    assert np.all(vol > 0) and np.all(np.isfinite(vol))


# ---- find_boundary_samples ------------------------------------------------------------------
@pytest.mark.parametrize("x, found", [(1.0, True), (1000.0, False)])
def test_find_boundary_samples_near_and_distant_fluid_particle(oracle, cube, x, found):
    b = _static(oracle, cube)
    b.initialize(KERNEL_SUPPORT_RADIUS, WEIGHTING)
    b.find_boundary_samples(KERNEL_SUPPORT_RADIUS, [[x, 0, 0]], SPACING)
    assert (b.neighbor_count(0, 0) > 0) == found


# ---- forces and steps -----------------------------------------------------------------------
def test_force_onto_boundary_moves_dynamic_boundary_center_of_mass(oracle, cube):
    b = _dynamic(oracle, cube)
    b.initialize(KERNEL_SUPPORT_RADIUS, WEIGHTING)
    before = b.samples(0)[3]
    b.add_force(0, [1000, 0, 0], before)
    b.step(0.1)
    assert b.samples(0)[3][0] > before[0]


def test_add_force_onto_boundary_accelerates_a_dynamic_boundary(oracle, cube):
    b = _dynamic(oracle, cube)
    b.step(0.0)
    b.add_force(0, [0, -100, 0], b.samples(0)[3])
    b.step(1.0)
    assert b.samples(0)[1][0][1] < 0.0


def test_add_force_onto_boundary_ignores_out_of_range_id(oracle, cube):
    b = _static(oracle, cube)
    b.add_force(5, [1, 0, 0], [0, 0, 0])
    assert len(b) == 1


def test_step_forward_in_time_is_noop_for_static_boundary(oracle, cube):
    b = _static(oracle, cube)
    b.initialize(KERNEL_SUPPORT_RADIUS, WEIGHTING)
    before = b.samples(0)[0]
    b.step(1.0)
    assert np.array_equal(b.samples(0)[0], before)


def test_step_forward_in_time_translates_a_moving_dynamic_boundary(oracle, cube):
    b = _dynamic(oracle, cube, (0, 0, 0), (1, 0, 0))
    b.step(0.0)
    before = b.samples(0)[0][0]
    b.step(1.0)
    assert np.linalg.norm(b.samples(0)[0][0] - before - [1, 0, 0]) < 1e-9


def test_dynamic_boundary_sample_velocities_match_rigid_body_formula_with_offset_com(oracle, cube):
    com, linear, omega = np.array([5.0, 0, 0]), np.array([0.5, 0, 0]), np.array([0, 0, 2.0])
    b = _dynamic(oracle, cube, com, linear, omega)
    b.step(0.0)
    pos, vel, _, c = b.samples(0)
    assert np.linalg.norm(c - com) < 1e-9
    want = linear + np.cross(omega, pos - com)
    assert np.all(np.linalg.norm(vel - want, axis=1) < 1e-9)
    assert np.all(np.linalg.norm(pos - com, axis=1) > 0.5)


def test_step_forward_in_time_rotates_samples_about_the_center_of_mass(oracle, cube):
    com = np.array([5.0, 0, 0])
    b = _dynamic(oracle, cube, com, (0, 0, 0), (0, 0, 2))
    b.step(0.0)
    p0 = b.samples(0)[0]
    b.step(0.25)
    p1 = b.samples(0)[0]
    assert np.all(np.abs(np.linalg.norm(p1 - com, axis=1) - np.linalg.norm(p0 - com, axis=1)) < 1e-9)
    assert np.all(np.abs(p1[:, 2] - p0[:, 2]) < 1e-9)
    assert np.abs(p1 - p0).max() > 0.1  # it did turn
