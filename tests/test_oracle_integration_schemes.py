"""Pins the oracle's integration schemes to the reference's unit tests:
EulerCromer (simulation_lib/tests/sph/integration_schemes/euler_cromer.rs:88-226)
and TakePredicted (tests/sph/integration_schemes/take_predicted.rs:66-219),
restated with the same inputs, expectations and tolerances. The reference's
fluids there hold a few sampled particles of which the tests set and read the
first one or two; the restatement does the same with three particles.

The trait-bound tests (Default and Clone impls) have nothing to restate.
"""
import numpy as np

N = 3


def _state(pos0=(0, 0, 0), vel0=(0, 0, 0), acc0=(0, 0, 0)):
    rng = np.random.default_rng(7)
    pos, vel, acc = (rng.normal(size=(N, 3)) for _ in range(3))
    pos[0], vel[0], acc[0] = pos0, vel0, acc0
    return pos, vel, acc


def _close(a, b, eps):
    assert np.linalg.norm(np.asarray(a) - np.asarray(b)) < eps, (a, b)


# ---- EulerCromer ----------------------------------------------------------------------------
def test_euler_cromer_single_particle_matches_semi_implicit_euler_update(oracle):
    pos0, vel0, acc0, dt = np.array([1.0, 2, 3]), np.array([0.5, -0.5, 1.0]), np.array([2.0, 0, -9.81]), 0.1
    pos, vel, _ = oracle.integrate_probe("EulerCromer", *_state(pos0, vel0, acc0), dt)
    v = vel0 + dt * acc0
    _close(vel[0], v, 1e-9)
    _close(pos[0], pos0 + dt * v, 1e-9)


def test_euler_cromer_position_update_uses_the_new_velocity_not_the_old_one(oracle):
    pos, _, _ = oracle.integrate_probe("EulerCromer", *_state((0, 0, 0), (1, 0, 0), (10, 0, 0)), 1.0)
    _close(pos[0], [11, 0, 0], 1e-9)
    assert np.linalg.norm(pos[0] - [1, 0, 0]) > 1e-3


def test_euler_cromer_zero_acceleration_reduces_to_straight_line_motion(oracle):
    vel0 = np.array([2.0, -1.0, 0.5])
    pos, vel, _ = oracle.integrate_probe("EulerCromer", *_state((0, 0, 0), vel0, (0, 0, 0)), 0.3)
    _close(vel[0], vel0, 1e-9)
    _close(pos[0], 0.3 * vel0, 1e-9)


def test_euler_cromer_zero_time_step_leaves_position_and_velocity_unchanged(oracle):
    pos0, vel0 = np.array([4.0, -2.0, 1.0]), np.array([1.0, 2.0, 3.0])
    pos, vel, _ = oracle.integrate_probe("EulerCromer", *_state(pos0, vel0, (-5, 0, 9.81)), 0.0)
    assert np.array_equal(vel[0], vel0)
    assert np.array_equal(pos[0], pos0)


def test_euler_cromer_does_not_modify_acceleration(oracle):
    acc0 = np.array([3.0, -4.0, 5.0])
    _, _, acc = oracle.integrate_probe("EulerCromer", *_state(acc0=acc0), 0.05)
    assert np.array_equal(acc[0], acc0)


def test_euler_cromer_works_without_integrator_slots(oracle):
    # no slot pool at all (EulerCromer::POSITION_SLOTS = VELOCITY_SLOTS = 0)
    oracle.integrate_probe("EulerCromer", *_state((1, 1, 1), (0.2, 0.3, 0.4), (1, 0, 0)), 0.1)


def test_euler_cromer_multiple_particles_are_updated_independently(oracle):
    pos, vel, acc = _state()
    pos[:2] = [(0, 0, 0), (5, 5, 5)]
    vel[:2] = [(1, 0, 0), (0, -2, 0)]
    acc[:2] = [(1, 0, 0), (0, 0, 3)]
    want_v = vel[:2] + 0.2 * acc[:2]
    want_x = pos[:2] + 0.2 * want_v
    p, v, _ = oracle.integrate_probe("EulerCromer", pos, vel, acc, 0.2)
    for i in range(2):
        _close(v[i], want_v[i], 1e-9)
        _close(p[i], want_x[i], 1e-9)


def test_euler_cromer_repeated_steps_under_constant_acceleration_match_the_manual_recurrence(oracle):
    g, dt = np.array([0.0, 0.0, -9.81]), 0.01
    x, v = np.zeros(3), np.zeros(3)
    for _ in range(5):
        v = v + dt * g
        x = x + dt * v
    st = _state(acc0=g)
    for _ in range(5):
        st = oracle.integrate_probe("EulerCromer", *st, dt)
    _close(st[1][0], v, 1e-9)
    _close(st[0][0], x, 1e-9)


# ---- TakePredicted --------------------------------------------------------------------------
def _slots():
    rng = np.random.default_rng(11)
    return rng.normal(size=(N, 3)), rng.normal(size=(N, 3))


def test_take_predicted_position_becomes_the_old_predicted_position(oracle):
    sp, sv = _slots()
    sp[0] = (9, 8, 7)
    pos, _, _, _ = oracle.integrate_probe("TakePredicted", *_state(), 0.1, sp, sv)
    assert np.array_equal(pos[0], [9, 8, 7])


def test_take_predicted_velocity_becomes_the_old_predicted_velocity(oracle):
    sp, sv = _slots()
    sv[0] = (1, -2, 3)
    _, vel, _, _ = oracle.integrate_probe("TakePredicted", *_state(), 0.1, sp, sv)
    assert np.array_equal(vel[0], [1, -2, 3])


def test_take_predicted_slots_hold_the_pre_step_current_state_after_committing(oracle):
    sp, sv = _slots()
    sp[0], sv[0] = (9, 9, 9), (9, 9, 9)
    _, _, _, (p_slot, v_slot) = oracle.integrate_probe("TakePredicted", *_state((1, 2, 3), (0.5, 0.5, 0.5)),
                                                       0.1, sp, sv)
    assert np.array_equal(p_slot[0], [1, 2, 3])
    assert np.array_equal(v_slot[0], [0.5, 0.5, 0.5])


def test_take_predicted_result_is_independent_of_dt(oracle):
    def run(dt):
        sp, sv = _slots()
        sp[0], sv[0] = (3, 3, 3), (4, 4, 4)
        return oracle.integrate_probe("TakePredicted", *_state((1, 1, 1), (2, 2, 2)), dt, sp, sv)
    a, b = run(0.001), run(1000.0)
    assert np.array_equal(a[0][0], b[0][0])
    assert np.array_equal(a[1][0], b[1][0])


def test_take_predicted_does_not_modify_acceleration(oracle):
    acc0 = np.array([3.0, -4.0, 5.0])
    _, _, acc, _ = oracle.integrate_probe("TakePredicted", *_state(acc0=acc0), 0.05, *_slots())
    assert np.array_equal(acc[0], acc0)


def test_take_predicted_multiple_particles_are_updated_independently(oracle):
    sp, sv = _slots()
    sp[:2] = [(1, 0, 0), (0, 2, 0)]
    sv[:2] = [(1, 0, 0), (0, 2, 0)]
    pos, vel, _, _ = oracle.integrate_probe("TakePredicted", *_state(), 0.1, sp, sv)
    assert np.array_equal(pos[0], [1, 0, 0]) and np.array_equal(vel[0], [1, 0, 0])
    assert np.array_equal(pos[1], [0, 2, 0]) and np.array_equal(vel[1], [0, 2, 0])


def test_take_predicted_repeated_calls_each_commit_whatever_was_predicted_since_the_last_call(oracle):
    sp, sv = _slots()
    sp[0], sv[0] = (1, 0, 0), (1, 0, 0)
    pos, vel, acc, (sp, sv) = oracle.integrate_probe("TakePredicted", *_state(), 0.1, sp, sv)
    assert np.array_equal(pos[0], [1, 0, 0])
    sp[0], sv[0] = (2, 0, 0), (2, 0, 0)
    pos, vel, acc, (sp, sv) = oracle.integrate_probe("TakePredicted", pos, vel, acc, 0.1, sp, sv)
    assert np.array_equal(pos[0], [2, 0, 0])
    assert np.array_equal(sp[0], [1, 0, 0])
