"""Pins the oracle's RigidBodyMotion to the reference's unit tests
(simulation_lib/tests/sph/boundary_handling/rigid_body_motion.rs:44-642),
restated one for one with the same inputs, expectations and tolerances.

The engine integrates the same body on the device (body_step); its two-way
coupling is checked against this oracle in the GPU parity tests, so these pins
are what ties the device's rigid motion to the reference's.
"""
import math

import numpy as np

FRAC_PI_2 = math.pi / 2


def _init(mass=1.0, I=(1.0, 1.0, 1.0), com=(0, 0, 0), q=(1, 0, 0, 0), v=(0, 0, 0), w=(0, 0, 0), I_inv=None):
    Ib = np.diag(I)
    Iinv = np.linalg.inv(Ib) if I_inv is None else np.diag(I_inv)
    return np.concatenate([[mass], Ib.ravel(), Iinv.ravel(), com, q, v, w]).astype(np.float64)


def _axis_angle(axis, angle):
    a = np.asarray(axis, np.float64)
    a = a / np.linalg.norm(a)
    return np.concatenate([[math.cos(angle / 2)], math.sin(angle / 2) * a])


def _checkpoint(com=(0, 0, 0), q=(1, 0, 0, 0), v=(0, 0, 0), L=(0, 0, 0), f=(0, 0, 0), t=(0, 0, 0)):
    return np.concatenate([com, q, v, L, f, t]).astype(np.float64)


def _close(a, b, eps):
    assert np.linalg.norm(np.asarray(a) - np.asarray(b)) < eps, (a, b)


def _angle(q):
    """Rotation angle of a unit quaternion (w, i, j, k) in [0, pi]."""
    w = abs(q[0])
    return 2.0 * math.atan2(np.linalg.norm(q[1:]), w)


# ---- construction, pose ---------------------------------------------------------------------
def test_new_computes_angular_momentum_from_inertia_and_angular_velocity(oracle):
    st = oracle.rigid_probe(_init(I=(2, 3, 4), I_inv=(0.5, 1 / 3, 0.25), w=(1, 2, 3)), "state")
    _close(st[10:13], [2, 6, 12], 1e-12)
    _close(st[19:22], [1, 2, 3], 1e-12)


def test_pose_combines_translation_and_orientation(oracle):
    body = _init(com=(1, 2, 3), q=_axis_angle((0, 0, 1), FRAC_PI_2))
    _close(oracle.rigid_probe(body, "local_to_world", (0, 0, 0)), [1, 2, 3], 1e-9)
    _close(oracle.rigid_probe(body, "local_to_world", (1, 0, 0)), [1, 3, 3], 1e-9)


def test_world_to_local_is_inverse_of_local_to_world(oracle):
    body = _init(com=(-2, 5, 0.5), q=_axis_angle((1, 1, 0), 1.234))
    p = np.array([3.0, -1.0, 2.0])
    _close(oracle.rigid_probe(body, "world_to_local", oracle.rigid_probe(body, "local_to_world", p)), p, 1e-9)
    _close(oracle.rigid_probe(body, "local_to_world", oracle.rigid_probe(body, "world_to_local", p)), p, 1e-9)


def test_local_to_world_vector_ignores_translation(oracle):
    q = _axis_angle((0, 0, 1), FRAC_PI_2)
    a = oracle.rigid_probe(_init(q=q), "local_to_world_vector", (1, 0, 0))
    b = oracle.rigid_probe(_init(com=(100, -50, 3), q=q), "local_to_world_vector", (1, 0, 0))
    _close(a, b, 1e-9)


# ---- velocity_at_point ----------------------------------------------------------------------
def test_velocity_at_cm_equals_linear_velocity(oracle):
    _close(oracle.rigid_probe(_init(v=(3, 4, 5)), "state")[7:10], [3, 4, 5], 1e-12)


def test_velocity_at_point_matches_rigid_body_formula(oracle):
    body = _init(v=(1, 0, 0), w=(0, 0, 2))
    _close(oracle.rigid_probe(body, "velocity_at_point", (1, 0, 0)), [1, 2, 0], 1e-12)


def test_velocity_at_point_uses_com_as_pivot_not_world_origin(oracle):
    body = _init(com=(5, 0, 0), w=(0, 0, 1))
    _close(oracle.rigid_probe(body, "velocity_at_point", (6, 0, 0)), [0, 1, 0], 1e-12)


def test_velocity_at_point_reduces_to_linear_velocity_at_the_com(oracle):
    v_lin, com = (-1.5, 0.25, 3.0), (5.0, -2.0, 1.0)
    body = _init(com=com, v=v_lin, w=(0.3, -0.7, 1.1))
    _close(oracle.rigid_probe(body, "velocity_at_point", com), v_lin, 1e-12)
    _close(oracle.rigid_probe(body, "velocity_at_point", oracle.rigid_probe(body, "state")[0:3]), v_lin, 1e-12)


def test_velocity_at_point_superposes_translation_and_rotation_off_origin(oracle):
    body = _init(com=(5, 0, 0), v=(0, 0, 2), w=(0, 0, 1))
    _close(oracle.rigid_probe(body, "velocity_at_point", (6, 0, 0)), [0, 1, 2], 1e-12)


def test_velocity_at_point_is_antisymmetric_in_the_lever_arm(oracle):
    com = np.array([1.0, -4.0, 2.5])
    body = _init(com=com, v=(0.7, 0, -0.2), w=(0.4, -1.3, 0.9))
    r = np.array([2.0, 0.5, -1.5])
    vp = oracle.rigid_probe(body, "velocity_at_point", com + r)
    vm = oracle.rigid_probe(body, "velocity_at_point", com - r)
    _close(0.5 * (vp + vm), oracle.rigid_probe(body, "state")[7:10], 1e-12)


def test_velocity_at_point_is_unaffected_along_the_rotation_axis(oracle):
    com, omega = np.array([-3.0, 2.0, 7.0]), np.array([0.0, 0.0, 2.5])
    body = _init(com=com, w=omega)
    _close(oracle.rigid_probe(body, "velocity_at_point", com + omega * 3.0), [0, 0, 0], 1e-12)


def test_velocity_field_satisfies_the_rigidity_constraint(oracle):
    body = _init(com=(2, -1, 0.5), q=_axis_angle((0, 1, 0), 0.83), v=(1, -2, 0.4), w=(0.6, 1.4, -0.9))
    a, b = np.array([4.0, 0.0, -2.0]), np.array([-1.0, 3.5, 1.0])
    rel = oracle.rigid_probe(body, "velocity_at_point", a) - oracle.rigid_probe(body, "velocity_at_point", b)
    assert abs(rel @ (a - b)) < 1e-11


def test_velocity_at_point_crosses_world_frame_angular_velocity(oracle):
    body = _init(I=(1, 2, 3), I_inv=(1, 0.5, 1 / 3), com=(1, 1, 1))
    ck = _checkpoint(com=(1, 1, 1), q=_axis_angle((0, 0, 1), FRAC_PI_2), L=(0, 1, 0))
    omega = oracle.rigid_probe(body, "state", restore=ck)[19:22]
    probe = np.array([1.0, 1.0, 1.0]) + np.array([1.0, 0.0, 0.0])
    got = oracle.rigid_probe(body, "velocity_at_point", probe, restore=ck)
    _close(got, np.cross(omega, [1, 0, 0]), 1e-12)
    _close(omega, [0, 1, 0], 1e-9)


# ---- add_force, reset_forces, checkpoint staging --------------------------------------------
def test_add_force_accumulates_force_and_torque(oracle):
    st = oracle.rigid_probe(_init(), "state", forces=[(1, 0, 0), (0, 1, 0)], locations=[(1, 0, 0), (1, 0, 0)])
    _close(st[13:16], [1, 1, 0], 1e-12)
    _close(st[16:19], [0, 0, 1], 1e-12)


def test_reset_forces_clears_pending_force_and_torque(oracle):
    st = oracle.rigid_probe(_init(), "state", forces=[(1, 0, 0)], locations=[(1, 0, 0)], reset=True)
    _close(st[13:16], [0, 0, 0], 1e-12)
    _close(st[16:19], [0, 0, 0], 1e-12)


def test_get_checkpoint_captures_pending_force_before_step(oracle):
    st = oracle.rigid_probe(_init(), "state", forces=[(4, 0, 0)], locations=[(0, 0, 0)])
    _close(st[13:16], [4, 0, 0], 1e-12)


# ---- step_forward_in_time -------------------------------------------------------------------
def test_step_forward_in_time_integrates_linear_motion_semi_implicitly(oracle):
    st = oracle.rigid_probe(_init(mass=2.0), "state", forces=[(4, 0, 0)], locations=[(0, 0, 0)], dt=0.1,
                            n_steps=1)
    _close(st[7:10], [0.2, 0, 0], 1e-12)
    _close(st[0:3], [0.02, 0, 0], 1e-12)


def test_step_forward_in_time_resets_forces(oracle):
    st = oracle.rigid_probe(_init(), "state", forces=[(1, 0, 0)], locations=[(0, 0, 0)], dt=0.1, n_steps=1)
    _close(st[13:16], [0, 0, 0], 1e-12)
    _close(st[16:19], [0, 0, 0], 1e-12)


def test_step_forward_in_time_conserves_angular_velocity_without_torque(oracle):
    for n in range(1, 6):
        st = oracle.rigid_probe(_init(w=(0, 0, 2)), "state", dt=0.01, n_steps=n)
        _close(st[19:22], [0, 0, 2], 1e-12)


def test_step_forward_in_time_rotates_orientation_approximately_as_expected(oracle):
    dt = 0.001
    q = oracle.rigid_probe(_init(w=(0, 0, 2)), "state", dt=dt, n_steps=1)[3:7]
    assert abs(_angle(q) - 2 * dt) < 1e-4
    axis = q[1:] / np.linalg.norm(q[1:]) * np.sign(q[0])
    _close(axis, [0, 0, 1], 1e-9)


def test_velocity_field_pivot_tracks_the_com_across_steps(oracle):
    body = _init(v=(1, 0, 0), w=(0, 0, 1))
    for n in range(1, 51):
        com = oracle.rigid_probe(body, "state", dt=0.01, n_steps=n)[0:3]
        got = oracle.rigid_probe(body, "velocity_at_point", com + np.array([1.0, 0, 0]), dt=0.01, n_steps=n)
        _close(got, [1, 1, 0], 1e-10)
    assert abs(com[0] - 0.5) < 1e-10


def test_orientation_integration_preserves_the_full_rotation_angle(oracle):
    q = oracle.rigid_probe(_init(w=(0, 0, 1)), "state", dt=0.5, n_steps=1)[3:7]
    assert abs(_angle(q) - 0.5) < 1e-12
    scaled_axis = q[1:] / np.linalg.norm(q[1:]) * np.sign(q[0]) * _angle(q)
    _close(scaled_axis, [0, 0, 0.5], 1e-12)


def test_orientation_integration_has_no_cumulative_angle_deficit(oracle):
    q = oracle.rigid_probe(_init(w=(0, 0, 2 * math.pi)), "state", dt=1e-3, n_steps=1000)[3:7]
    assert abs(_angle(q)) < 1e-11


# ---- checkpoint / restore -------------------------------------------------------------------
def test_checkpoint_roundtrip_preserves_full_state(oracle):
    a = _init(com=(1, 2, 3), q=_axis_angle((0, 0, 1), 0.5), v=(0.1, 0.2, 0.3), w=(0.4, 0.5, 0.6))
    sa = oracle.rigid_probe(a, "state", forces=[(1, 0, 0)], locations=[(1, 2, 3)])
    sb = oracle.rigid_probe(_init(), "state", restore=sa[:19])
    _close(sb[0:3], sa[0:3], 1e-12)
    _close(sb[7:10], sa[7:10], 1e-12)
    _close(sb[19:22], sa[19:22], 1e-12)
    _close(sb[13:16], sa[13:16], 1e-12)
    _close(sb[16:19], sa[16:19], 1e-12)


def test_restore_from_checkpoint_refreshes_derived_state_for_new_orientation(oracle):
    body = _init(I=(1, 2, 3), I_inv=(1, 0.5, 1 / 3))
    ck = _checkpoint(q=_axis_angle((0, 0, 1), FRAC_PI_2), L=(1, 1, 0))
    _close(oracle.rigid_probe(body, "state", restore=ck)[19:22], [0.5, 1.0, 0.0], 1e-9)


def test_restore_from_checkpoint_preserves_pending_force_for_next_step(oracle):
    ck = _checkpoint(f=(4, 0, 0))
    st = oracle.rigid_probe(_init(mass=2.0), "state", restore=ck, dt=0.1, n_steps=1)
    _close(st[7:10], [0.2, 0, 0], 1e-12)
