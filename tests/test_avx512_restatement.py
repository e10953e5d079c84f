"""The AVX-512 CPU restatement (oracle/ap26_avx512.c) against the plain
oracle and the pinned reference reports.  CPU only; skipped on a CPU
without AVX-512 VBMI2."""
import ctypes
import glob
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN

c64 = ctypes.c_int64


def vp(a):
    return a.ctypes.data_as(ctypes.c_void_p)


@pytest.fixture(scope="module")
def a5(oracle):
    if not oracle.a5_supported():
        pytest.skip("CPU without AVX-512 VBMI2")
    return oracle


@pytest.mark.parametrize("K,shift,f0,f1", [
    (366384, 0, 0, 2 * 443555),                       # first n43 values
    (44121555, 640, 10 ** 9 + 17, 10 ** 9 + 400_017),  # ragged, mid-lattice
    (1, 15360, 4_808_136_200 - 300_000, 4_808_136_200),  # end of the lattice, largest SHIFT
    (400_000_000, 1280, 2_000_000_000, 2_000_250_000),   # largest K in the domain
    # 61*67*71*73: all four primes of the two pair strings divide K, so each
    # bans one residue instead of 24 (the densest searchable K)
    (21182921, 640, 3_000_000_000, 3_000_300_000),
    (61 * 67 * 30, 0, 123_456, 423_456),                # 61*67 | K (a searchable K)
])
def test_a5_sieve_equals_oracle(a5, K, shift, f0, f1):
    cap = 1 << 20
    a, pos, b = np.zeros(cap, np.int64), np.zeros(cap, np.uint64), np.zeros(cap, np.int64)
    n_o = a5.ao_sieve(K, shift, c64(f0), c64(f1), vp(a), vp(pos), c64(cap), None, 4)
    n_a = a5.a5_sieve(K, shift, c64(f0), c64(f1), vp(b), c64(cap), 4)
    assert n_o == n_a > 0
    assert np.array_equal(np.sort(a[:n_o]), np.sort(b[:n_a]))


def test_a5_search_finds_pinned_reference_reports(a5):
    """Slices around reports of the reference's own search (oracle pins):
    the same (k, first) at the same lattice position, and the same output as
    the plain oracle's search over the slice."""
    for path in sorted(glob.glob(os.path.join(GOLDEN, "oracle_pin_*.json"))):
        p = json.load(open(path))
        K, shift = p["K"], p["shift"]
        for r in p["reports"][:4]:
            f0, f1 = r["f"] - 40, r["f"] + 40
            cap = 64
            ks, fs, ns = np.zeros(cap, np.int32), np.zeros(cap, np.int64), np.zeros(cap, np.int64)
            pos = np.zeros(cap, np.uint64)
            n = a5.a5_search(K, shift, c64(f0), c64(f1), vp(ks), vp(fs), vp(ns), vp(pos),
                             c64(cap), None, 2)
            got = {(int(pos[i]), int(ks[i]), int(fs[i])) for i in range(n)}
            want = ((r["f"] << 10) | (r["w"] << 6) | r["b"], r["k"], r["first"])
            assert want in got, (K, r)
            ks2, fs2, pos2 = np.zeros(cap, np.int32), np.zeros(cap, np.int64), np.zeros(cap, np.uint64)
            n2 = a5.ao_search(K, shift, c64(f0), c64(f1), vp(ks2), vp(fs2), vp(pos2), c64(cap),
                              None, 1)
            assert got == {(int(pos2[i]), int(ks2[i]), int(fs2[i])) for i in range(n2)}
