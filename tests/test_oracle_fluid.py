"""Pins the oracle's Fluid bookkeeping to the reference's unit tests
(simulation_lib/tests/sph/fluid.rs:130-308): swap-remove disabling, the
`id < num_active` assertion, drop_inactive and resize_slots. The engine's
disabled-particle order is checked against this oracle on the GPU, so these
pins tie the engine's renumbering to the reference's.

The checkpoint conversions of the same file are format tests and are restated
against the engine's checkpoint encoders; reconstruct_surfaces of an empty
fluid is pinned with the surface reconstruction.
"""
import numpy as np
import pytest


def _three():
    return [[1.0, 0, 0], [2.0, 0, 0], [3.0, 0, 0]], [1.0, 2.0, 3.0]


def test_fluid_disable_decreases_active_count(oracle):
    r = oracle.fluid_probe(*_three(), disable=[1])
    assert r["len"] == 2 and r["total_len"] == 3


def test_fluid_disable_swaps_with_last_active(oracle):
    r = oracle.fluid_probe(*_three(), disable=[0])
    assert np.array_equal(r["position"][0], [3, 0, 0]) and r["mass"][0] == 3.0
    assert np.array_equal(r["position"][2], [1, 0, 0])


def test_fluid_disable_swaps_fluid_id(oracle):
    r = oracle.fluid_probe(*_three(), fluid_ids=[10, 20, 30], disable=[0])
    assert r["fluid_id"][0] == 30 and r["fluid_id"][2] == 10


def test_fluid_disable_last_active_no_swap(oracle):
    r = oracle.fluid_probe([[1.0, 0, 0], [2.0, 0, 0]], [1.0, 2.0], disable=[1])
    assert r["len"] == 1 and np.array_equal(r["position"][0], [1, 0, 0])


@pytest.mark.parametrize("ids", [[1], [0, 0]])
def test_fluid_disable_out_of_range_or_after_all_disabled_fails(oracle, ids):
    # the reference panics on `assert!(id < self.num_active)`
    with pytest.raises(IndexError):
        oracle.fluid_probe([[1.0, 0, 0]], [1.0], disable=ids)


def test_fluid_drop_inactive(oracle):
    r = oracle.fluid_probe(*_three(), disable=[1], drop=True)
    assert r["total_len"] == 2 and r["len"] == 2
    assert r["position"].shape == (2, 3) and r["mass"].shape == (2,)


def test_fluid_disable_all(oracle):
    r = oracle.fluid_probe([[1.0, 0, 0], [2.0, 0, 0]], [1.0, 2.0], disable=[0, 0])
    assert r["len"] == 0 and r["total_len"] == 2


def test_resize_slots_creates_the_requested_pools_sized_to_total_len(oracle):
    r = oracle.fluid_probe([[1.0, 0, 0], [2.0, 0, 0]], [1.0, 1.0], slots=[1, 2, 0, 1])
    assert r["slot_counts"] == [1, 2, 0, 1] and r["slot_len"] == 2


def test_resize_slots_with_all_zero_counts_leaves_pools_empty(oracle):
    r = oracle.fluid_probe([[1.0, 0, 0]], [1.0], slots=[0, 0, 0, 0])
    assert r["slot_counts"] == [0, 0, 0, 0] and r["slot_len"] == 0


def test_disabling_keeps_slots_sized_and_drop_truncates_them(oracle):
    # slots follow the particles through swap and truncate (fluid.rs:166-204)
    r = oracle.fluid_probe(*_three(), slots=[1, 1, 1, 1], disable=[0])
    assert r["slot_len"] == 3
    r = oracle.fluid_probe(*_three(), slots=[1, 1, 1, 1], disable=[0], drop=True)
    assert r["slot_len"] == 2
