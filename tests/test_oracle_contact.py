"""The oracle's rigid-rigid contact (VolumeMapBoundary, volume_map_boundary.rs:
55-1102, 1440-1453) on small volume-map scenes.

The reference has no known-answer tests for its contact solver, so this
restatement is unpinned; these tests hold it to the properties the solver
is built for (Probst & Teschner's contact LCP as the reference's comments
describe it): no contact cells without an overlap of both bodies' solids or
without bounding boxes, contact pressures that push overlapping bodies
apart (equal and opposite for a symmetric pair), support against gravity on
a static floor, and friction inside the Coulomb cone.
"""
import numpy as np
import pytest

from conftest import oracle_config

SPACING = 0.01
H = 2 * SPACING
DT = 1e-3


def _ball(oracle, radius):
    from sphgpu import scenes
    v, f = scenes.icosphere(2, radius)
    sdf, _ = oracle.build_fields(v, f, 4 * SPACING, H, sdf_only=True)
    return sdf, v


def _plate(oracle, half):
    from sphgpu import scenes
    v = scenes.CUBE_VERTICES * np.asarray(half)
    sdf, _ = oracle.build_fields(v, scenes.CUBE_FACES_OUTWARD, 4 * SPACING, H, sdf_only=True)
    return sdf, v


def _system(oracle, bodies):
    """bodies: [(sdf, mesh vertices in the body frame, RigidInit or None)]; a
    lone fluid particle far away keeps the system valid."""
    from sphgpu import scenes
    sc = scenes.Scene(
        procedures={"integration_scheme": "EulerCromer", "pressure_solver": "SESPH",
                    "boundary_handling": "VolumeMapBoundary"},
        parameters={"rest_density_grid_spacing": SPACING, "kernel_support_radius": H,
                    "disable_particles_below": -50.0, "fluid_viscosity": 0.0, "boundary_viscosity": 0.0,
                    "boundary_pressure_acceleration_weighting": 0.7, "boundary_rest_volume_weighting": 1.0,
                    "stiffness": 1000.0, "time_increment": DT},
        cfl_time_step=False, position=np.array([[5.0, 5.0, 5.0]]), mass=np.array([1e-3]))
    s = oracle.OracleSystem(oracle_config(sc))
    s.upload_fluid(sc.position, sc.velocity, sc.mass, sc.fluid_id)
    for sdf, verts, rigid in bodies:
        s.add_volume_map_boundary(sdf, sdf, None if rigid is None else rigid.to_array32())
    s.initialize()
    for bi, (sdf, verts, rigid) in enumerate(bodies):
        lo, hi = verts.min(0), verts.max(0)
        s.set_vm_aabb(bi, 0.5 * (lo + hi), 0.5 * (hi - lo))
    return s


def _rigid(center, v=(0, 0, 0), w=(0, 0, 0), mass=1.0, inertia=1e-3):
    from sphgpu.system import RigidInit
    return RigidInit(mass=mass, inertia_body=np.eye(3) * inertia, center_of_mass=center,
                     linear_velocity=v, angular_velocity=w)


def test_no_cells_without_overlap_or_bounding_boxes(oracle):
    sdf, v = _ball(oracle, 0.06)
    s = _system(oracle, [(sdf, v, _rigid((0.0, 0.0, 0.0))), (sdf, v, _rigid((0.2, 0.0, 0.0)))])
    f, t, cells, _ = s.contact_probe(DT, 2)
    assert cells == 0 and not f.any() and not t.any()


def test_overlapping_balls_are_pushed_apart_symmetrically(oracle):
    sdf, v = _ball(oracle, 0.06)
    s = _system(oracle, [(sdf, v, _rigid((-0.055, 0.0, 0.0))), (sdf, v, _rigid((0.055, 0.0, 0.0)))])
    f, t, cells, its = s.contact_probe(DT, 2)
    assert cells > 0
    # gravity acts on both; the contact forces are along x and opposite, up to
    # the discretized SDF: its lattice (dx = 4 cm, nodes every 1.3 cm) is not
    # centered on the ball and is coarse against the 1 cm overlap
    assert f[0, 0] < 0 < f[1, 0]
    assert abs(f[0, 0] + f[1, 0]) < 1e-2 * abs(f[0, 0])
    assert np.abs(f[:, 1:]).max() < 0.1 * abs(f[0, 0])


def test_ball_on_a_static_plate_is_held_against_gravity(oracle):
    ball, vb = _ball(oracle, 0.05)
    plate, vp = _plate(oracle, (0.15, 0.15, 0.02))
    mass = 0.5
    # the plate spans z in [-0.02, 0.02]; the ball's bottom dips 5 mm into it
    # while falling at 0.1 m/s
    s = _system(oracle, [(plate, vp, None),
                         (ball, vb, _rigid((0.0, 0.0, 0.065), v=(0.0, 0.0, -0.1), mass=mass))])
    f, t, cells, its = s.contact_probe(DT, 2)
    assert cells > 0
    # the contact force stops the approach: it exceeds the weight plus the
    # momentum the ball would carry into the plate within one step
    assert f[1, 2] > mass * 9.81
    assert f[0, 2] < 0  # the reaction on the plate, which is static and does not move



def test_friction_stays_inside_the_cone(oracle):
    ball, vb = _ball(oracle, 0.05)
    plate, vp = _plate(oracle, (0.15, 0.15, 0.02))
    other, _ = _ball(oracle, 0.05)
    # a ball sliding along x over a second, resting ball below it
    s = _system(oracle, [(ball, vb, _rigid((0.0, 0.0, 0.0), mass=2.0)),
                         (other, vb, _rigid((0.01, 0.0, 0.095), v=(0.5, 0.0, -0.05), mass=0.5))])
    f, t, cells, its = s.contact_probe(DT, 2)
    assert cells > 0
    n = np.array([0.01, 0.0, 0.095])
    n /= np.linalg.norm(n)
    fn = f[1] @ n
    ft = np.linalg.norm(f[1] - fn * n)
    assert fn > 0
    assert ft <= 0.5 * fn * 1.5  # friction coefficient 0.5; the cone is taken per contact cell
    assert f[1, 0] < 0  # friction opposes the sliding
