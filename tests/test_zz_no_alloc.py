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


def _noalloc(L, torch, rng_, pos, samples):
    dpos = torch.from_numpy(np.ascontiguousarray(pos, np.float64)).cuda()
    dsmp = torch.from_numpy(np.ascontiguousarray(samples, np.float64)).cuda()
    n, ns = pos.shape[0], samples.shape[0]
    doff = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
    total = C.c_size_t()
    rc = L.sph_spatial_hashing_find_samples_noalloc(rng_, n, C.c_void_p(dpos.data_ptr()), ns,
                                                    C.c_void_p(dsmp.data_ptr()), C.c_void_p(doff.data_ptr()),
                                                    None, 0, C.byref(total), 0)
    assert rc == 6  # SPH_ERR_CAPACITY: sizes the output first
    didx = torch.zeros(max(total.value, 1), dtype=torch.int32, device="cuda")
    rc = L.sph_spatial_hashing_find_samples_noalloc(rng_, n, C.c_void_p(dpos.data_ptr()), ns,
                                                    C.c_void_p(dsmp.data_ptr()), C.c_void_p(doff.data_ptr()),
                                                    C.c_void_p(didx.data_ptr()), didx.numel(), C.byref(total), 0)
    assert rc == 0, L.sph_last_error()
    off = doff.cpu().numpy().astype(np.uint64)
    idx = didx.cpu().numpy().astype(np.uint32)[:total.value]
    return off, idx


def test_noalloc_find_samples_matches_allocating_entry_point_twice():
    torch = pytest.importorskip("torch")
    from sphgpu import _capi, find_samples
    L = _capi.load()
    rng = np.random.default_rng(11)
    cases = []
    for n, ns, spread in ((4000, 3000, 0.5), (2500, 5000, 0.8)):
        pos = rng.uniform(-spread, spread, size=(n, 3)).astype(np.float32).astype(np.float64)
        smp = rng.uniform(-spread, spread, size=(ns, 3))
        smp[:5] = pos[:5] + np.array([0.1, 0.0, 0.0])  # pairs exactly at the range
        cases.append((pos, smp))
    for pos, smp in cases:  # two calls in a row on the shared static array
        off_s, idx_s = _noalloc(L, torch, 0.1, pos, smp)
        off_a, idx_a = find_samples(0.1, pos, smp)
        assert np.array_equal(off_s, off_a)
        assert np.array_equal(idx_s, idx_a)


def test_noalloc_rejects_sizes_beyond_the_static_array():
    from sphgpu import _capi
    L = _capi.load()
    total = C.c_size_t()
    rc = L.sph_spatial_hashing_find_samples_noalloc(0.1, 10, C.c_void_p(16), (1 << 20) + 1, C.c_void_p(16),
                                                    C.c_void_p(16), None, 0, C.byref(total), 0)
    assert rc == 1
    assert b"at most 1048576" in L.sph_last_error()
