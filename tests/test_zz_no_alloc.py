"""The allocation-free neighbor search entry point.

sph_spatial_hashing_find_samples_noalloc serves callers that cannot allocate
device memory themselves through the library (their allocator belongs to
another runtime or pool, or their loop forbids allocation): they pass device
buffers they already own, and the library keeps its temporaries in one
static device array. This checks, through the C ABI, that two calls in a row
(the array keeps the previous call's contents) give exactly the neighbor
lists of the allocating entry point. It sits in its own file, collected last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(L, torch, rng_, pos, samples, capacity=None):
    """Calls the entry point twice: once to size the output, then with an
    index buffer of `capacity` entries (default: exactly the total)."""
    dpos = torch.from_numpy(np.ascontiguousarray(pos, np.float64)).cuda()
    dsmp = torch.from_numpy(np.ascontiguousarray(samples, np.float64)).cuda()
    n, ns = pos.shape[0], samples.shape[0]
    doff = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
    total = C.c_size_t()
    rc = L.sph_spatial_hashing_find_samples_noalloc(rng_, n, C.c_void_p(dpos.data_ptr() if n else None), ns,
                                                    C.c_void_p(dsmp.data_ptr() if ns else None),
                                                    C.c_void_p(doff.data_ptr()), None, 0, C.byref(total), 0)
    if total.value == 0:
        assert rc in (0, 6)
    else:
        assert rc == 6  # SPH_ERR_CAPACITY: sizes the output first
    cap = total.value if capacity is None else capacity
    didx = torch.zeros(max(cap, 1), dtype=torch.int32, device="cuda")
    rc = L.sph_spatial_hashing_find_samples_noalloc(rng_, n, C.c_void_p(dpos.data_ptr() if n else None), ns,
                                                    C.c_void_p(dsmp.data_ptr() if ns else None),
                                                    C.c_void_p(doff.data_ptr()), C.c_void_p(didx.data_ptr()), cap,
                                                    C.byref(total), 0)
    if cap < total.value:
        assert rc == 6, L.sph_last_error()
        return None, None
    assert rc == 0, L.sph_last_error()
    off = doff.cpu().numpy().astype(np.uint64)
    idx = didx.cpu().numpy().astype(np.uint32)[:total.value]
    return off, idx


def _cases():
    rng = np.random.default_rng(11)
    cases = []
    for n, ns, spread in ((4000, 3000, 0.5), (2500, 5000, 0.8)):
        pos = rng.uniform(-spread, spread, size=(n, 3)).astype(np.float32).astype(np.float64)
        smp = rng.uniform(-spread, spread, size=(ns, 3))
        smp[:5] = pos[:5] + np.array([0.1, 0.0, 0.0])  # pairs exactly at the range
        cases.append((pos, smp))
    # spread over 160 cells per axis: cells 64 apart share a bucket of the
    # fixed 2^18-bucket table, so buckets mix samples of several cells
    pos = rng.uniform(-8.0, 8.0, size=(6000, 3)).astype(np.float32).astype(np.float64)
    smp = np.concatenate([rng.uniform(-8.0, 8.0, size=(6000, 3)), pos[:3000] + 0.03])
    cases.append((pos, smp))
    # every sample in one cell: one bucket holds all of them, in index order
    smp = rng.uniform(0.2001, 0.2999, size=(20000, 3))
    pos = rng.uniform(0.1, 0.4, size=(300, 3))
    cases.append((pos, smp))
    return cases


def test_noalloc_find_samples_matches_allocating_entry_point_twice():
    torch = pytest.importorskip("torch")
    from sphgpu import _capi, find_samples
    L = _capi.load()
    for pos, smp in _cases():  # two calls in a row on the shared static array
        off_a, idx_a = find_samples(0.1, pos, smp)
        for _ in range(2):
            off_s, idx_s = _noalloc(L, torch, 0.1, pos, smp)
            assert np.array_equal(off_s, off_a)
            assert np.array_equal(idx_s, idx_a)


def test_noalloc_empty_inputs_and_short_capacity():
    torch = pytest.importorskip("torch")
    from sphgpu import _capi, find_samples
    L = _capi.load()
    rng = np.random.default_rng(3)
    pos = rng.uniform(-0.3, 0.3, size=(500, 3))
    smp = rng.uniform(-0.3, 0.3, size=(800, 3))
    # no samples: every row is empty
    off_s, idx_s = _noalloc(L, torch, 0.1, pos, np.zeros((0, 3)))
    off_a, idx_a = find_samples(0.1, pos, np.zeros((0, 3)))
    assert np.array_equal(off_s, off_a) and idx_s.size == 0 and off_s[-1] == 0
    # no positions: offsets hold the single leading zero
    off_s, idx_s = _noalloc(L, torch, 0.1, np.zeros((0, 3)), smp)
    assert off_s.tolist() == [0] and idx_s.size == 0
    # a non-zero capacity below the total is refused with the total reported
    off_a, idx_a = find_samples(0.1, pos, smp)
    assert idx_a.size > 10
    assert _noalloc(L, torch, 0.1, pos, smp, capacity=idx_a.size - 1) == (None, None)
    # and the next call with room still gives the allocating entry point's rows
    off_s, idx_s = _noalloc(L, torch, 0.1, pos, smp)
    assert np.array_equal(off_s, off_a) and np.array_equal(idx_s, idx_a)


def test_noalloc_rejects_sizes_beyond_the_static_array():
    from sphgpu import _capi
    L = _capi.load()
    total = C.c_size_t()
    rc = L.sph_spatial_hashing_find_samples_noalloc(0.1, 10, C.c_void_p(16), (1 << 20) + 1, C.c_void_p(16),
                                                    C.c_void_p(16), None, 0, C.byref(total), 0)
    assert rc == 1
    assert b"at most 1048576" in L.sph_last_error()
