#!/usr/bin/env python3
"""Generate golden raw-AP fixtures from the reference CPU build.

Test infrastructure.  Runs ``oracle/_ref/ref_harness raw K SHIFT`` (the
reference's own Search_avx2, compiled from its sources by
``oracle/build_ref.sh``) for every searchable K of a range and writes the raw
reports -- every ``ReportSolution(k, K, first)`` call the search makes, in the
reference's order (src/cpu/cpuavx2.cpp:551) -- to
``tests/golden/ref_raw/shift<SHIFT>/<K>.txt``, one ``k K first`` line each,
followed by a trailer line ``# n=<count> seconds=<t>``.

A whole K costs the reference about 550-620 s on one core, so this is run
once, here, and the fixtures are committed.

Usage:
  python tests/golden/make_golden.py --ks 366384 44121555 47715109 --shift 0
  python tests/golden/make_golden.py --kmin 43241056 --count 64 --shift 0 -j 6
"""
import argparse
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")


def will_search(k):
    """src/common/AP26.cpp:649-653: K is skipped if divisible by 29..59."""
    return all(k % p for p in (29, 31, 37, 41, 43, 47, 53, 59))


def run_one(k, shift, outdir):
    path = os.path.join(outdir, f"{k}.txt")
    if os.path.exists(path):
        return k, "cached"
    out = subprocess.run([HARNESS, "raw", str(k), str(shift)], check=True,
                         capture_output=True, text=True).stdout
    lines, secs, n = [], None, None
    for ln in out.splitlines():
        if ln.startswith("R "):
            lines.append(ln[2:])
        elif ln.startswith("DONE "):
            _, _k, n, secs, _isa = ln.split()
    assert n is not None and int(n) == len(lines), (k, n, len(lines))
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        f.write("\n".join(lines) + ("\n" if lines else ""))
        f.write(f"# n={len(lines)} seconds={secs}\n")
    os.replace(tmp, path)
    return k, f"{len(lines)} reports in {secs}s"


def copy_reference_tests(ref_root="/root/reference"):
    """The reference's own golden SOL files (tests/TEST-<K>.txt: the SOL line
    and result hash of `AP26 K K 0`) become tests/golden/TEST-<K>.txt."""
    import shutil
    for name in sorted(os.listdir(os.path.join(ref_root, "tests"))):
        if name.startswith("TEST-") and name.endswith(".txt"):
            shutil.copyfile(os.path.join(ref_root, "tests", name), os.path.join(HERE, name))
            print("copied", name)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--copy-tests", action="store_true",
                    help="copy the reference's tests/TEST-*.txt golden files")
    ap.add_argument("--ks", type=int, nargs="*", default=[])
    ap.add_argument("--kmin", type=int)
    ap.add_argument("--count", type=int, default=0)
    ap.add_argument("--shift", type=int, default=0)
    ap.add_argument("-j", "--jobs", type=int, default=4)
    a = ap.parse_args()
    if a.copy_tests:
        copy_reference_tests()
    ks = list(a.ks)
    if a.kmin is not None:
        ks += list(range(a.kmin, a.kmin + a.count))
    ks = [k for k in ks if will_search(k)]
    outdir = os.path.join(HERE, "ref_raw", f"shift{a.shift}")
    os.makedirs(outdir, exist_ok=True)
    if not os.access(HARNESS, os.X_OK):
        sys.exit(f"missing {HARNESS}: run oracle/build_ref.sh first")
    with ThreadPoolExecutor(a.jobs) as ex:
        for k, msg in ex.map(lambda k: run_one(k, a.shift, outdir), ks):
            print(k, msg, flush=True)


if __name__ == "__main__":
    main()
