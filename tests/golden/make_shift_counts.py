#!/usr/bin/env python3
"""Generate tests/golden/shift_counts.json: whole-K sieve survivor counts
(after the 7..23 filter) at nonzero SHIFT, for every K with a recorded
reference raw-report file under tests/golden/ref_raw/shift<SHIFT>/.
Computed by the AVX-512 CPU restatement (oracle/ap26_avx512.c), which the
test suite checks against the plain oracle on slices; the plain oracle is
pinned to the reference's known survivor count at SHIFT 0.  Test
infrastructure; about 80 s per K on 8 cores.
"""
import ctypes
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
N59_PER_K = 4808136200


def main():
    L = ctypes.CDLL(os.path.join(ROOT, "oracle", "liboracle.so"))
    L.a5_sieve.restype = ctypes.c_int64
    if not L.a5_supported():
        sys.exit("needs a CPU with AVX-512 VBMI2")
    threads = os.cpu_count() or 1
    out = []
    raw = os.path.join(HERE, "ref_raw")
    for d in sorted(os.listdir(raw)):
        shift = int(d[5:])
        if shift == 0:
            continue
        for name in sorted(os.listdir(os.path.join(raw, d))):
            K = int(name[:-4])
            t0 = time.time()
            n = L.a5_sieve(K, shift, ctypes.c_int64(0), ctypes.c_int64(N59_PER_K), None,
                           ctypes.c_int64(0), threads)
            assert n > 0
            out.append({"K": K, "shift": shift, "candidates": n})
            print(K, shift, n, f"{time.time() - t0:.0f}s", flush=True)
    with open(os.path.join(HERE, "shift_counts.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
