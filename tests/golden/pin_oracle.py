#!/usr/bin/env python3
"""Pin the oracle: full-K oracle searches vs the reference's own outputs.

Test infrastructure.  For each K given, runs the oracle's whole-K search
(oracle/ap26_oracle.c ao_search, all 10 shift words) and writes
``tests/golden/oracle_pin_<K>_<SHIFT>.json`` with the candidate count and
every raw report (k, first, candidate n, AVX2 order key) in the reference's
AVX2 order.  It then checks, and records in the file, that

  * the report list equals the reference's raw ReportSolution sequence
    (tests/golden/ref_raw/shift<SHIFT>/<K>.txt, produced by the reference
    Search_avx2 itself), element by element;
  * for K=366384 SHIFT=0 the candidate count equals the reference's known
    answer 38,838,420 (src/opencl/AP26.h:343).

Usage: python tests/golden/pin_oracle.py 366384 44121555 47715109 [-t THREADS]
"""
import argparse
import ctypes
import json
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
N59_PER_K = 4808136200
KNOWN_SURVIVORS = {(366384, 0): 38838420}


def load_oracle():
    L = ctypes.CDLL(os.path.join(ROOT, "oracle", "liboracle.so"))
    L.ao_search.restype = ctypes.c_int64
    L.ao_avx2_order_key.restype = ctypes.c_uint64
    L.ao_avx2_order_key.argtypes = [ctypes.c_uint64]
    return L


def read_ref_raw(K, shift):
    path = os.path.join(HERE, "ref_raw", f"shift{shift}", f"{K}.txt")
    out = []
    for ln in open(path):
        if ln.startswith("#"):
            continue
        k, KK, first = map(int, ln.split())
        out.append((k, KK, first))
    return out


def oracle_search(L, K, shift, f0, f1, threads, cap=1 << 16):
    ks = np.zeros(cap, np.int32)
    firsts = np.zeros(cap, np.int64)
    pos = np.zeros(cap, np.uint64)
    ncand = ctypes.c_int64(0)
    n = L.ao_search(K, shift, ctypes.c_int64(f0), ctypes.c_int64(f1),
                    ks.ctypes.data_as(ctypes.c_void_p), firsts.ctypes.data_as(ctypes.c_void_p),
                    pos.ctypes.data_as(ctypes.c_void_p), ctypes.c_int64(cap),
                    ctypes.byref(ncand), threads)
    assert 0 <= n <= cap, n
    MOD = 258559632607830
    reps = []
    for i in range(n):
        p = int(pos[i])
        f, w, b = p >> 10, (p >> 6) & 15, p & 63
        reps.append({"k": int(ks[i]), "first": int(firsts[i]), "f": f, "w": w, "b": b,
                     "key": int(L.ao_avx2_order_key(p))})
    reps.sort(key=lambda r: r["key"])
    return reps, ncand.value


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("ks", type=int, nargs="+")
    ap.add_argument("--shift", type=int, default=0)
    ap.add_argument("-t", "--threads", type=int, default=os.cpu_count())
    a = ap.parse_args()
    L = load_oracle()
    for K in a.ks:
        t0 = time.time()
        reps, ncand = oracle_search(L, K, a.shift, 0, N59_PER_K, a.threads)
        secs = time.time() - t0
        ref = read_ref_raw(K, a.shift)
        mine = [(r["k"], K, r["first"]) for r in reps]
        rec = {
            "K": K, "shift": a.shift, "candidates": ncand, "reports": reps, "seconds": secs,
            "matches_reference_raw": mine == ref,
            "reference_raw_count": len(ref),
        }
        if (K, a.shift) in KNOWN_SURVIVORS:
            rec["known_survivors"] = KNOWN_SURVIVORS[(K, a.shift)]
            rec["matches_known_survivors"] = ncand == KNOWN_SURVIVORS[(K, a.shift)]
        out = os.path.join(HERE, f"oracle_pin_{K}_{a.shift}.json")
        with open(out, "w") as f:
            json.dump(rec, f, indent=0)
        print(K, "candidates", ncand, "reports", len(reps), "match_ref", mine == ref,
              "secs %.0f" % secs, flush=True)


if __name__ == "__main__":
    main()
