#!/usr/bin/env python3
"""Generate tests/golden/report_vectors.txt: the reference's own
ReportSolution (src/common/AP26.cpp:549-602) on single raw reports, run by
oracle/_ref/ref_report (built from the reference sources by
oracle/build_ref.sh).  Test infrastructure.

Cases: progressions of difference K*23# around base-2 strong pseudoprimes
that fail the 9-base validation (composite Mersenne numbers 2^p - 1,
p = 11..59, and 2^32 + 1) -- one-term reports, [prime, spsp],
[prime, spsp, prime], [spsp, prime, prime]; 3825123056546413051, a composite
that passes all nine bases, alone and after a prime; golden APs and their
sub-progressions; reports that are not base-2 APs (the reference exits);
a term past 2^62 (exits); empty reports; start hashes near MAXINTV; and a
seeded sample of recorded raw reports.

Each line: k K first h0 status hash sols
  status  ok | exit      (exit = the reference ended the process)
  hash    result_hash after the call (- on exit)
  sols    len:first,... solutions in SOL order (- if none)
"""
import os
import random
import subprocess
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
TOOL = os.path.join(ROOT, "oracle", "_ref", "ref_report")
P23 = 223092870
BASES = (2, 3, 5, 7, 11, 13, 17, 19, 23)
SPSP2 = [2 ** p - 1 for p in (11, 23, 29, 37, 41, 43, 47, 53, 59)] + [2 ** 32 + 1]
PSP9 = 3825123056546413051


def sprp(a, n):
    d, t = n - 1, 0
    while d % 2 == 0:
        d //= 2
        t += 1
    x = pow(a, d, n)
    if x in (1, n - 1):
        return True
    for _ in range(t - 1):
        x = x * x % n
        if x == n - 1:
            return True
    return False


def prime9(n):
    return all(sprp(b, n) for b in BASES)


def cases():
    out = []
    for s in SPSP2:
        assert sprp(2, s) and not prime9(s)
        out += [(1, 1, s, 0), (1, 366384, s, 0)]
        got = {}
        for K in range(1, 4000):
            D = K * P23
            if s - D > 23 and "pre" not in got and prime9(s - D):
                got["pre"] = K
            if s - D > 23 and "mid" not in got and prime9(s - D) and prime9(s + D):
                got["mid"] = K
            if "post" not in got and prime9(s + D) and prime9(s + 2 * D):
                got["post"] = K
            if len(got) == 3:
                break
        if "pre" in got:
            out.append((2, got["pre"], s - got["pre"] * P23, 0))
        if "mid" in got:
            out.append((3, got["mid"], s - got["mid"] * P23, 0))
            out.append((3, got["mid"], s - got["mid"] * P23, 1999999000))
        if "post" in got:
            out.append((3, got["post"], s, 0))
    assert sprp(2, PSP9) and prime9(PSP9)
    out.append((1, 5, PSP9, 0))
    for K in range(1, 200):
        if prime9(PSP9 - K * P23):
            out.append((2, K, PSP9 - K * P23, 0))
            break
    first, K = 6171054912832631, 366384          # the 25-term AP of TEST-366384.txt
    D = K * P23
    out += [(25, K, first, 0), (24, K, first + D, 0), (20, K, first + 5 * D, 0),
            (25, K, first, 1999999900), (25, K, first, 2000000000),
            (26, K, first, 0), (26, K, first - D, 0), (19, K, first + 6 * D, 0),
            (0, 7, 1000000007, 0), (0, 5, 10 ** 12, 0), (3, 5, 10 ** 12, 0),
            (1, 5, (1 << 62) + 1, 0)]
    rng = random.Random(26)
    raw_dir = os.path.join(HERE, "ref_raw", "shift0")
    raw = []
    for name in sorted(os.listdir(raw_dir)):
        with open(os.path.join(raw_dir, name)) as f:
            raw += [tuple(map(int, ln.split())) for ln in f if not ln.startswith("#")]
    for k, KK, fi in rng.sample(raw, 40):
        out.append((k, KK, fi, rng.choice([0, 12345, 1999999500])))
    return out


def run(k, K, first, h0):
    with tempfile.TemporaryDirectory() as d:
        p = subprocess.run([TOOL, str(k), str(K), str(first), str(h0)], cwd=d,
                           capture_output=True, text=True)
    sols = [ln.split()[1:] for ln in p.stdout.splitlines() if ln.startswith("Solution: ")]
    sol = ",".join(f"{a}:{c}" for a, _, c in sols) or "-"
    if p.returncode != 0:
        return "exit", "-", "-"
    h = [ln.split()[1] for ln in p.stdout.splitlines() if ln.startswith("HASH ")][0]
    return "ok", h, sol


def main():
    lines = ["# k K first h0 status hash sols  -- reference ReportSolution via oracle/_ref/ref_report"]
    for k, K, first, h0 in cases():
        st, h, sol = run(k, K, first, h0)
        lines.append(f"{k} {K} {first} {h0} {st} {h} {sol}")
    with open(os.path.join(HERE, "report_vectors.txt"), "w") as f:
        f.write("\n".join(lines) + "\n")
    print(f"{len(lines) - 1} vectors")


if __name__ == "__main__":
    main()
