"""The allocation-free entry point, ap26_sieve_count_noalloc.

It serves callers that cannot allocate device memory themselves (a host
framework owns the memory pool, a plugin host forbids cudaMalloc/cudaFree
because they synchronise the device, or the caller must not fail on memory
exhaustion mid-run): they pass device buffers they already own, and all of
the entry point's scratch lives in a fixed device array inside the library.

Checked through the C ABI against the allocating entry point
(ap26_sieve_count) on two calls in a row, the second with fewer K than the
first so stale counts from the first call would show.  The counts are
integers: equality is exact.  This file sorts last so that a stop-at-first-
failure run has executed every other test before it; it also passes alone in
a fresh process (the first call sets the device up itself).
"""
import ctypes

import pytest

import ap26_b200 as A

pytestmark = pytest.mark.gpu


def _noalloc(Ks, shift):
    import torch
    d_k = torch.tensor(Ks, dtype=torch.int32, device="cuda")
    d_out = torch.full((len(Ks),), -7, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = A.lib.ap26_sieve_count_noalloc(0, ctypes.c_void_p(d_k.data_ptr()), len(Ks), shift,
                                        ctypes.c_void_p(d_out.data_ptr()),
                                        ctypes.c_void_p(stream))
    assert rc == A.OK, A.lib.ap26_strerror(rc)
    torch.cuda.synchronize()
    return d_out.cpu().tolist()


def test_noalloc_counts_match_allocating_entry_point_twice():
    import torch
    torch.cuda.init()
    first = [366384, 1000037, 43241056]
    second = [44121555]
    shift = 640
    got1 = _noalloc(first, shift)
    got2 = _noalloc(second, shift)
    ctx = A.Context(0)
    try:
        exp1, _ = ctx.sieve_count(first, shift)
        exp2, _ = ctx.sieve_count(second, shift)
    finally:
        ctx.close()
    assert got1 == exp1.tolist()
    assert got2 == exp2.tolist()
    assert min(got1 + got2) > 0


def test_noalloc_rejects_sizes_beyond_its_maximum():
    import torch
    d_k = torch.ones(65, dtype=torch.int32, device="cuda")
    d_out = torch.zeros(65, dtype=torch.int64, device="cuda")
    rc = A.lib.ap26_sieve_count_noalloc(0, ctypes.c_void_p(d_k.data_ptr()), 65, 0,
                                        ctypes.c_void_p(d_out.data_ptr()), None)
    assert rc == A.E_CAPACITY
