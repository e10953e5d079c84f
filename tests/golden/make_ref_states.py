#!/usr/bin/env python3
"""Generate tests/golden/ref_states.txt: the checkpoints the reference CPU
build writes while it searches the golden K (oracle/_ref/AP26, built from the
reference sources by oracle/build_ref.sh; AVX2 dispatch on this host).
Test infrastructure.

The reference writes "KMIN KMAX SHIFT K ITER result_hash last_trickle" to
AP26-state.{a,b}.txt (AP26.cpp:360-394) before each 4-word pass of a K
(ITER 0, 4, 8) and after the workunit (K = KMAX + 1).  Every distinct
(K, ITER, result_hash) state seen while the search runs is recorded; the
hash at (K, ITER) covers the reports of shift words 0..ITER-1 of K.  Runs
the three golden K concurrently, about ten minutes.

Each line: KMIN KMAX SHIFT K ITER result_hash
"""
import os
import shutil
import subprocess
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
TOOL = os.path.join(ROOT, "oracle", "_ref", "AP26")
KS = (366384, 44121555, 47715109)


def read_states(d):
    out = []
    for name in ("AP26-state.a.txt", "AP26-state.b.txt"):
        try:
            with open(os.path.join(d, name)) as f:
                parts = f.read().split()
        except OSError:
            continue
        if len(parts) >= 6:
            out.append(tuple(int(x) for x in parts[:6]))
    return out


def main():
    runs = []
    for K in KS:
        d = tempfile.mkdtemp(prefix=f"ref_states_{K}_")
        p = subprocess.Popen([TOOL, str(K), str(K), "0"], cwd=d, stdout=subprocess.DEVNULL,
                             stderr=subprocess.DEVNULL)
        runs.append((K, d, p, set()))
    while any(p.poll() is None for _, _, p, _ in runs):
        for _, d, _, seen in runs:
            seen.update(read_states(d))
        time.sleep(0.2)
    lines = ["# KMIN KMAX SHIFT K ITER result_hash  -- states written by oracle/_ref/AP26 K K 0"]
    for K, d, p, seen in runs:
        assert p.returncode == 0, K
        seen.update(read_states(d))
        with open(os.path.join(d, "SOL-AP26.txt")) as f, \
                open(os.path.join(HERE, f"TEST-{K}.txt")) as g:
            assert f.read() == g.read(), K
        for s in sorted(seen, key=lambda t: (t[3], t[4])):
            lines.append(" ".join(map(str, s)))
        shutil.rmtree(d)
    with open(os.path.join(HERE, "ref_states.txt"), "w") as f:
        f.write("\n".join(lines) + "\n")
    print("\n".join(lines))


if __name__ == "__main__":
    main()
