"""CPU tests that pin the oracle (oracle/ap26_oracle.c) to the reference:
its report/hash restatement against the reference's golden SOL files, its
SPRP against the reference's strong_prp verdicts, its whole-K search against
the reference's raw reports and survivor known answer, and its sieve against
a direct restatement of the reference's OKOK lookups."""
import ctypes
import glob
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, GOLDEN_KS, golden_sol, ref_raw


def oracle_sol(oracle, K, raw):
    h = ctypes.c_int(0)
    sol = ctypes.create_string_buffer(1 << 16)
    for k, KK, first in raw:
        assert oracle.ao_report(ctypes.byref(h), k, KK, ctypes.c_int64(first), sol, len(sol)) == 0
    hexb = ctypes.create_string_buffer(17)
    oracle.ao_hash_hex(K, K, h, hexb)
    return sol.value.decode() + hexb.value.decode() + "\n"


@pytest.mark.parametrize("K", GOLDEN_KS)
def test_oracle_report_matches_golden(oracle, K):
    assert oracle_sol(oracle, K, ref_raw(K)) == golden_sol(K)


def test_oracle_report_matches_reference_report_vectors(oracle):
    """ao_report against the reference's own ReportSolution on single raw
    reports (tests/golden/report_vectors.txt): splits around base-2
    pseudoprimes, the 9-base-passing composite, exits and hash wrap-around."""
    n_exit = 0
    with open(os.path.join(GOLDEN, "report_vectors.txt")) as f:
        for ln in f:
            if ln.startswith("#"):
                continue
            k, K, first, h0, st, h, sols = ln.split()
            hh = ctypes.c_int(int(h0))
            buf = ctypes.create_string_buffer(1 << 12)
            rc = oracle.ao_report(ctypes.byref(hh), int(k), int(K), ctypes.c_int64(int(first)),
                                  buf, len(buf))
            if st == "exit":
                assert rc < 0, ln
                n_exit += 1
                continue
            assert rc == 0 and hh.value == int(h), ln
            got = [f"{x.split()[0]}:{x.split()[2]}" for x in buf.value.decode().splitlines()]
            assert (",".join(got) or "-") == sols, ln
    assert n_exit >= 4


def sprp_vectors():
    out = []
    with open(os.path.join(GOLDEN, "sprp_vectors.txt")) as f:
        for ln in f:
            if ln.startswith("#"):
                continue
            n, a, v = map(int, ln.split())
            out.append((n, a, v))
    return out


def test_oracle_sprp_matches_reference_strong_prp(oracle):
    vec = sprp_vectors()
    assert len(vec) > 1000
    for n, a, v in vec:
        assert oracle.ao_sprp(ctypes.c_int64(n), ctypes.c_int64(a)) == v, (n, a)


def pins():
    files = sorted(glob.glob(os.path.join(GOLDEN, "oracle_pin_*.json")))
    return [json.load(open(f)) for f in files]


def test_oracle_whole_k_pins():
    """Recorded full-K oracle searches (tests/golden/pin_oracle.py) equal the
    reference's raw report sequence; K=366384 has 38,838,420 survivors."""
    ps = pins()
    if not ps:
        pytest.skip("no oracle pin files recorded")
    for p in ps:
        assert p["matches_reference_raw"], p["K"]
        assert len(p["reports"]) == p["reference_raw_count"]
        if "known_survivors" in p:
            assert p["candidates"] == p["known_survivors"]


def test_oracle_reproduces_pinned_reports_locally(oracle):
    """Re-run the oracle on the single lattice position of a few pinned
    reports: it must produce the same (k, first)."""
    ps = pins()
    if not ps:
        pytest.skip("no oracle pin files recorded")
    cap = 64
    for p in ps:
        for r in p["reports"][:6]:
            ks = np.zeros(cap, np.int32)
            fs = np.zeros(cap, np.int64)
            pos = np.zeros(cap, np.uint64)
            nc = ctypes.c_int64()
            n = oracle.ao_search(p["K"], p["shift"], ctypes.c_int64(r["f"]),
                                 ctypes.c_int64(r["f"] + 1), ks.ctypes.data_as(ctypes.c_void_p),
                                 fs.ctypes.data_as(ctypes.c_void_p),
                                 pos.ctypes.data_as(ctypes.c_void_p), ctypes.c_int64(cap),
                                 ctypes.byref(nc), 1)
            got = {(int(ks[i]), int(fs[i]), int(pos[i]) & 1023) for i in range(n)}
            assert (r["k"], r["first"], (r["w"] << 6) | r["b"]) in got


def test_oracle_sieve_equals_direct_table_restatement(oracle):
    """ao_sieve against a numpy restatement of cpusse2.cpp:434-594 (OKOK
    lookups ANDed for all 83 primes, then the 7..23 filter) on a slice."""
    K, shift = 366384, 640
    primes = [oracle.ao_prime(i) for i in range(83)]
    tabs = []
    for p in primes:
        t = np.zeros((10, p), np.uint64)
        for w in range(10):
            buf = (ctypes.c_uint64 * p)()
            oracle.ao_okok(K, shift + 64 * w, p, buf)
            t[w] = np.frombuffer(buf, np.uint64)
        tabs.append(t)
    f0, f1 = 1_000_000, 1_020_000
    n59 = np.array([oracle.ao_n59(K, ctypes.c_int64(f)) for f in range(f0, f1)], np.int64)
    MOD = 258559632607830
    exp = []
    for w in range(10):
        m = np.full(len(n59), np.uint64(0xFFFFFFFFFFFFFFFF))
        for i, p in enumerate(primes):
            m &= tabs[i][w][n59 % p]
        for idx in np.nonzero(m)[0]:
            mm = int(m[idx])
            for b in range(64):
                if mm >> b & 1:
                    n = int(n59[idx]) + (b + shift + 64 * w) * MOD
                    if all(n % q for q in (7, 11, 13, 17, 19, 23)):
                        exp.append(n)
    cap = 1 << 16
    cn = np.zeros(cap, np.int64)
    cp = np.zeros(cap, np.uint64)
    cons = ctypes.c_uint64()
    got = oracle.ao_sieve(K, shift, ctypes.c_int64(f0), ctypes.c_int64(f1),
                          cn.ctypes.data_as(ctypes.c_void_p), cp.ctypes.data_as(ctypes.c_void_p),
                          ctypes.c_int64(cap), ctypes.byref(cons), 2)
    assert got == len(exp)
    assert sorted(cn[:got].tolist()) == sorted(exp)


def test_oracle_n43_count_and_setup(oracle):
    out = (ctypes.c_int64 * 10840)()
    assert oracle.ao_n43(366384, out) == 10840
    s = (ctypes.c_int64 * 9)()
    oracle.ao_setup(366384, s)
    assert s[0] == 366384 * 223092870


def test_reference_survivor_counts_are_consistent():
    """tests/golden/ref_counts.json holds survivor counts counted in the
    reference's own search: K=366384 at SHIFT 0 is its known answer
    (src/opencl/AP26.h:343), and every entry's report count equals its
    recorded raw-report file."""
    import json
    import os
    d = json.load(open(os.path.join(GOLDEN, "ref_counts.json")))
    by = {(e["K"], e["shift"]): e for e in d}
    assert by[(366384, 0)]["survivors"] == 38838420
    assert len({s for _, s in by}) >= 3
    for (K, shift), e in by.items():
        assert len(ref_raw(K, shift)) == e["reports"], (K, shift)
        # a sieve prime p in 61..73 that divides K bans one residue instead
        # of 24: each such prime multiplies the survivors by about 1.5
        dense = sum(K % p == 0 for p in (61, 67, 71, 73))
        assert 30_000_000 < e["survivors"] < 70_000_000 * 1.6 ** dense
