#!/usr/bin/env python3
"""Generate golden fixtures from the reference CPU build.

Test infrastructure.  Runs ``oracle/_ref/ref_harness raw K SHIFT`` (the
reference's own Search_avx2, compiled from its sources by
``oracle/build_ref.sh``) and records, per (K, SHIFT):

* the raw reports -- every ``ReportSolution(k, K, first)`` call the search
  makes, in the reference's order (src/cpu/cpuavx2.cpp:551) -- in
  ``tests/golden/ref_raw/shift<SHIFT>/<K>.txt``, one ``k K first`` line each,
  then a trailer ``# n=<count> seconds=<t> survivors=<s>``;
* the sieve survivor count (candidates that start a chain walk, counted by
  the harness's PrimeQ wrapper) in ``tests/golden/ref_counts.json``.

A raw file that already exists is not rewritten; its reports are compared
with the new run instead (a mismatch aborts).  A whole K costs the reference
about 550-650 s on one core, so this is run once, here, and the fixtures are
committed.

Usage:
  python tests/golden/make_golden.py --ks 366384 44121555 47715109 --shift 0
  python tests/golden/make_golden.py --kmin 43241056 --count 64 --shift 0 -j 6
  python tests/golden/make_golden.py --pairs 28096782:1280 7928262:15360 -j 6
  python tests/golden/make_golden.py --bench-workloads -j 6
      (every (K, SHIFT) of bench.py's batched, serving and sieve-pair keys)
"""
import argparse
import json
import os
import subprocess
import sys
import threading
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")


def will_search(k):
    """src/common/AP26.cpp:649-653: K is skipped if divisible by 29..59."""
    return all(k % p for p in (29, 31, 37, 41, 43, 47, 53, 59))


COUNTS = os.path.join(HERE, "ref_counts.json")
_counts_lock = threading.Lock()


def load_counts():
    if not os.path.exists(COUNTS):
        return {}
    with open(COUNTS) as f:
        return {(e["K"], e["shift"]): e for e in json.load(f)}


def _store_count(k, shift, survivors, secs, n_reports):
    with _counts_lock:
        d = load_counts()
        d[(k, shift)] = {"K": k, "shift": shift, "survivors": survivors,
                         "reports": n_reports, "seconds": float(secs)}
        tmp = COUNTS + ".tmp"
        with open(tmp, "w") as f:
            json.dump([d[key] for key in sorted(d)], f, indent=1)
            f.write("\n")
        os.replace(tmp, COUNTS)


def run_one(k, shift):
    outdir = os.path.join(HERE, "ref_raw", f"shift{shift}")
    os.makedirs(outdir, exist_ok=True)
    path = os.path.join(outdir, f"{k}.txt")
    if os.path.exists(path) and (k, shift) in load_counts():
        return k, shift, "cached"
    out = subprocess.run([HARNESS, "raw", str(k), str(shift)], check=True,
                         capture_output=True, text=True).stdout
    lines, secs, n, survivors = [], None, None, None
    for ln in out.splitlines():
        if ln.startswith("R "):
            lines.append(ln[2:])
        elif ln.startswith("COUNT "):
            survivors = int(ln.split()[1])
        elif ln.startswith("DONE "):
            _, _k, n, secs, _isa = ln.split()
    assert n is not None and int(n) == len(lines) and survivors is not None, (k, n, len(lines))
    if os.path.exists(path):
        with open(path) as f:
            old = [ln.rstrip("\n") for ln in f if not ln.startswith("#")]
        assert old == lines, f"reference reports of K={k} SHIFT={shift} differ from {path}"
    else:
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            f.write("\n".join(lines) + ("\n" if lines else ""))
            f.write(f"# n={len(lines)} seconds={secs} survivors={survivors}\n")
        os.replace(tmp, path)
    _store_count(k, shift, survivors, secs, len(lines))
    return k, shift, f"{len(lines)} reports, {survivors} survivors in {secs}s"


def copy_reference_tests(ref_root):
    """The reference's own golden SOL files (tests/TEST-<K>.txt: the SOL line
    and result hash of `AP26 K K 0`) become tests/golden/TEST-<K>.txt."""
    import shutil
    for name in sorted(os.listdir(os.path.join(ref_root, "tests"))):
        if name.startswith("TEST-") and name.endswith(".txt"):
            shutil.copyfile(os.path.join(ref_root, "tests", name), os.path.join(HERE, name))
            print("copied", name)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--copy-tests", metavar="REFERENCE_ROOT",
                    help="copy the reference's tests/TEST-*.txt golden files from this tree")
    ap.add_argument("--ks", type=int, nargs="*", default=[])
    ap.add_argument("--kmin", type=int)
    ap.add_argument("--count", type=int, default=0)
    ap.add_argument("--shift", type=int, default=0)
    ap.add_argument("--pairs", nargs="*", default=[], help="K:SHIFT pairs")
    ap.add_argument("--bench-workloads", action="store_true",
                    help="every (K, SHIFT) of bench.py's secondary workloads")
    ap.add_argument("-j", "--jobs", type=int, default=4)
    a = ap.parse_args()
    if a.copy_tests:
        copy_reference_tests(a.copy_tests)
    ks = list(a.ks)
    if a.kmin is not None:
        ks += list(range(a.kmin, a.kmin + a.count))
    pairs = [(k, a.shift) for k in ks if will_search(k)]
    pairs += [tuple(map(int, p.split(":"))) for p in a.pairs]
    if a.bench_workloads:
        sys.path.insert(0, ROOT)
        import bench
        pairs += bench.fixture_pairs()
    if not os.access(HARNESS, os.X_OK):
        sys.exit(f"missing {HARNESS}: run oracle/build_ref.sh first")
    with ThreadPoolExecutor(a.jobs) as ex:
        for k, sh, msg in ex.map(lambda p: run_one(*p), pairs):
            print(k, sh, msg, flush=True)


if __name__ == "__main__":
    main()
