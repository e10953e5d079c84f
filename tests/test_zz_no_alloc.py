"""The allocation-free entry point, ap26_sieve_count_noalloc.

It serves callers that cannot allocate device memory themselves (a host
framework owns the memory pool, a plugin host forbids cudaMalloc/cudaFree
because they synchronise the device, or the caller must not fail on memory
exhaustion mid-run): they pass device buffers they already own, and all of
the entry point's scratch lives in a fixed device array inside the library.

Checked through the C ABI against the allocating entry point
(ap26_sieve_count) on two calls in a row, the second with fewer K than the
first so stale counts from the first call would show; against survivor
counts recorded from the reference itself (K=366384 at SHIFT 0 is the
reference's known answer, src/opencl/AP26.h:343); and with invalid K mixed
into a call, which must read -1 without disturbing the valid entries or
costing sieve time.  The counts are integers: equality is exact.  This file
sorts last so that a stop-at-first-failure run has executed every other test
before it; it also passes alone in a fresh process (the first call sets the
device up itself).
"""
import ctypes
import json
import os
import time

import pytest

import ap26_b200 as A
from conftest import GOLDEN

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


def test_noalloc_counts_equal_reference_survivor_counts():
    import torch
    torch.cuda.init()
    assert _noalloc([366384], 0) == [38838420]
    # counted in the reference's own search (tests/golden/ref_counts.json)
    pinned = json.load(open(os.path.join(GOLDEN, "ref_counts.json")))
    by_shift = {}
    for p in pinned:
        if p["shift"]:
            by_shift.setdefault(p["shift"], []).append(p)
    for shift, ps in sorted(by_shift.items())[:2]:
        ps = ps[:2]
        assert _noalloc([p["K"] for p in ps], shift) == [p["survivors"] for p in ps], shift


def test_noalloc_invalid_k_reads_minus_one_and_costs_no_sieve_time():
    import torch
    torch.cuda.init()
    good = 366384
    t0 = time.perf_counter()
    one = _noalloc([good], 0)
    t_one = time.perf_counter() - t0
    mixed = [0, good, A.KMAX_SAFE + 1, -5]
    t0 = time.perf_counter()
    got = _noalloc(mixed, 0)
    t_mixed = time.perf_counter() - t0
    assert one == [38838420]
    assert got == [-1, 38838420, -1, -1]
    # each invalid K used to cost a whole K of sieving; now only the valid one runs
    assert t_mixed < 1.5 * t_one + 0.05, (t_mixed, t_one)
    assert _noalloc([0, -1], 0) == [-1, -1]
