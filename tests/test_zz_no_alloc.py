"""GPU: v2m_bin_sort_noalloc, the hash's counting sort for callers that cannot
allocate device memory (their process keeps the GPU's memory in its own pool,
so a library cudaMalloc could fail or fragment it, and a cudaFree would stall
their streams). It works in a fixed scratch array of the library and the
caller's own buffers.

Through the C ABI, on two calls in a row with different inputs (the second
call must not see the first call's leftovers), its bin starts and sorted ids
equal the session's own hash build bit for bit (the tolerance of integer work);
random keys equal numpy's stable argsort; a crowded bin and a million keys in
one bin are ordered in linear time; a key outside [0, nbins) is refused, and the
next valid call is unaffected; requests beyond the scratch's fixed sizes are
refused with a clear error; a non-default stream works. The buffers here come
from torch: the test allocates, the entry point does not.
"""
import ctypes as C
import time

import numpy as np
import pytest

import cases
from trussnet_b200 import Session, _lib

pytestmark = pytest.mark.gpu

MAX_BINS = 1 << 20   # V2M_NOALLOC_MAX_BINS
MAX_KEYS = 1 << 22   # V2M_NOALLOC_MAX_KEYS


def session_sort(g, nd):
    with Session(g, cases.params(1), nd.copy()) as s:
        s.rebuild()
        return s.read("key"), s.read("sorted"), s.read("cstart"), s.nkeys[0]


def noalloc_call(L, key, nbins, stream=None):
    """One call on device buffers made here; returns (rc, sorted, cstart)."""
    import torch
    n = key.size
    dkey = torch.tensor(key, dtype=torch.int32, device="cuda")
    dsorted = torch.full((max(n, 1),), -1, dtype=torch.int32, device="cuda")
    dcstart = torch.full((nbins + 1,), -1, dtype=torch.int32, device="cuda")
    st = stream if stream is not None else torch.cuda.current_stream()
    torch.cuda.synchronize()
    rc = L.v2m_bin_sort_noalloc(dkey.data_ptr(), n, nbins, dsorted.data_ptr(), dcstart.data_ptr(),
                                C.c_void_p(st.cuda_stream))
    return rc, dsorted.cpu().numpy()[:n], dcstart.cpu().numpy()


def expected(key, nbins):
    order = np.argsort(key, kind="stable").astype(np.int32)
    cstart = np.zeros(nbins + 1, np.int32)
    cstart[1:] = np.cumsum(np.bincount(key, minlength=nbins))
    return order, cstart


def test_noalloc_sort_equals_session_build_twice(cuda_lib):
    L = _lib.load()
    inputs = [cases.shells_small(), cases.sphere_small()]
    for g, nd in inputs:   # two calls in a row, different sizes
        key, want_sorted, want_cstart, nkeys = session_sort(g, nd)
        assert nkeys + 1 <= MAX_BINS + 1
        rc, got_sorted, got_cstart = noalloc_call(L, key, nkeys)
        assert rc == 0, L.v2m_bin_sort_noalloc_error().decode()
        assert np.array_equal(got_cstart, want_cstart)
        assert np.array_equal(got_sorted, want_sorted)


def test_noalloc_random_and_crowded_keys(cuda_lib):
    """Random keys over more bins than are used, then keys crowding into a few
    bins (in-bin sorts above the one-thread size), each against numpy."""
    L = _lib.load()
    rng = np.random.default_rng(11)
    for n, nbins, skew in [(50_000, 300_000, False), (200_000, 4096, True), (3_000, 7, True)]:
        if skew:
            key = np.minimum(rng.geometric(0.3, n) - 1, nbins - 1).astype(np.int32)
        else:
            key = rng.integers(0, nbins, n, dtype=np.int32)
        rc, got_sorted, got_cstart = noalloc_call(L, key, nbins)
        assert rc == 0, L.v2m_bin_sort_noalloc_error().decode()
        want_sorted, want_cstart = expected(key, nbins)
        assert np.array_equal(got_cstart, want_cstart)
        assert np.array_equal(got_sorted, want_sorted)


def test_noalloc_one_bin_of_a_million_keys_is_linear(cuda_lib):
    """Every key in one bin: the in-bin order is one block's radix sort, done in
    well under a second (an insertion sort would take hours)."""
    L = _lib.load()
    n = 1 << 20
    key = np.zeros(n, np.int32)
    noalloc_call(L, key[:4096], 1)   # warm-up
    t0 = time.perf_counter()
    rc, got_sorted, got_cstart = noalloc_call(L, key, 1)
    dt = time.perf_counter() - t0
    assert rc == 0, L.v2m_bin_sort_noalloc_error().decode()
    assert np.array_equal(got_sorted, np.arange(n, dtype=np.int32))
    assert got_cstart.tolist() == [0, n]
    assert dt < 2.0, f"{dt:.2f} s for one bin of {n} keys"


def test_noalloc_bad_key_then_valid_call(cuda_lib):
    """A key equal to nbins is refused; the next valid call starts clean."""
    L = _lib.load()
    key = np.array([0, 3, 1, 4, 2], np.int32)
    rc, _, _ = noalloc_call(L, key, 4)
    assert rc == _lib.V2M_ERR_ARG
    assert b"outside [0, nbins)" in L.v2m_bin_sort_noalloc_error()
    key = np.array([3, 0, 3, 1, 0, 2, 3], np.int32)
    rc, got_sorted, got_cstart = noalloc_call(L, key, 4)
    assert rc == 0, L.v2m_bin_sort_noalloc_error().decode()
    want_sorted, want_cstart = expected(key, 4)
    assert np.array_equal(got_sorted, want_sorted) and np.array_equal(got_cstart, want_cstart)


def test_noalloc_on_a_side_stream(cuda_lib):
    import torch
    L = _lib.load()
    rng = np.random.default_rng(12)
    key = rng.integers(0, 1000, 20_000, dtype=np.int32)
    s = torch.cuda.Stream()
    rc, got_sorted, got_cstart = noalloc_call(L, key, 1000, stream=s)
    assert rc == 0, L.v2m_bin_sort_noalloc_error().decode()
    want_sorted, want_cstart = expected(key, 1000)
    assert np.array_equal(got_sorted, want_sorted) and np.array_equal(got_cstart, want_cstart)


def test_noalloc_rejects_sizes_beyond_its_scratch(cuda_lib):
    L = _lib.load()
    rc = L.v2m_bin_sort_noalloc(None, 0, MAX_BINS + 1, None, C.c_void_p(1), None)
    assert rc == _lib.V2M_ERR_ARG
    assert b"exceed the fixed scratch" in L.v2m_bin_sort_noalloc_error()
    rc = L.v2m_bin_sort_noalloc(C.c_void_p(1), MAX_KEYS + 1, 16, C.c_void_p(1), C.c_void_p(1), None)
    assert rc == _lib.V2M_ERR_ARG
    assert b"keys exceed the fixed scratch" in L.v2m_bin_sort_noalloc_error()
