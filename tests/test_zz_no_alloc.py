"""GPU: v2m_bin_sort_noalloc, the hash's counting sort for callers that cannot
allocate device memory (their process keeps the GPU's memory in its own pool,
so a library cudaMalloc could fail or fragment it, and a cudaFree would stall
their streams). It works in a fixed scratch array of the library and the
caller's own buffers.

Through the C ABI, on two calls in a row with different inputs (the second
call must not see the first call's leftovers), its bin starts and sorted ids
equal the session's own hash build bit for bit (the tolerance of integer work);
a request beyond the scratch's fixed size is refused with a clear error. The
buffers here come from torch: the test allocates, the entry point does not.
"""
import ctypes as C

import numpy as np
import pytest

import cases
from trussnet_b200 import Session, _lib

pytestmark = pytest.mark.gpu

MAX_BINS = 1 << 20   # V2M_NOALLOC_MAX_BINS


def session_sort(g, nd):
    with Session(g, cases.params(1), nd.copy()) as s:
        s.rebuild()
        return s.read("key"), s.read("sorted"), s.read("cstart"), s.nkeys[0]


def noalloc_sort(L, key, nkeys):
    import torch
    n = key.size
    dkey = torch.tensor(key, dtype=torch.int32, device="cuda")
    dsorted = torch.full((max(n, 1),), -1, dtype=torch.int32, device="cuda")
    dcstart = torch.full((nkeys + 1,), -1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    rc = L.v2m_bin_sort_noalloc(dkey.data_ptr(), n, nkeys, dsorted.data_ptr(), dcstart.data_ptr(),
                                C.c_void_p(stream))
    assert rc == 0, L.v2m_bin_sort_noalloc_error().decode()
    return dsorted.cpu().numpy()[:n], dcstart.cpu().numpy()


def test_noalloc_sort_equals_session_build_twice(cuda_lib):
    L = _lib.load()
    inputs = [cases.shells_small(), cases.sphere_small()]
    for g, nd in inputs:   # two calls in a row, different sizes
        key, want_sorted, want_cstart, nkeys = session_sort(g, nd)
        assert nkeys + 1 <= MAX_BINS + 1
        got_sorted, got_cstart = noalloc_sort(L, key, nkeys)
        assert np.array_equal(got_cstart, want_cstart)
        assert np.array_equal(got_sorted, want_sorted)


def test_noalloc_rejects_more_bins_than_its_scratch(cuda_lib):
    L = _lib.load()
    rc = L.v2m_bin_sort_noalloc(None, 0, MAX_BINS + 1, None, C.c_void_p(1), None)
    assert rc == _lib.V2M_ERR_ARG
    assert b"exceed the fixed scratch" in L.v2m_bin_sort_noalloc_error()
