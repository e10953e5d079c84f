"""Device-side ReportSolution (src/common/AP26.cpp:484-602) against the
reference's own ReportSolution on single reports (tests/golden/
report_vectors.txt), the oracle's restatement (oracle/ap26_oracle.c
ao_report) over every recorded raw report, and the golden SOL files; the
9-base strong-PRP test against verdicts of the reference's own strong_prp
(tests/golden/sprp_vectors.txt).

The vectors place base-2 strong pseudoprimes that fail the 9-base check
(composite Mersenne numbers 2^p - 1, p = 11..59, and 2^32 + 1) and
3825123056546413051, a composite that passes all nine validation bases, as
terms of short progressions of difference K*23#: they drive every branch of
the recursion (Non-Solution with leading and trailing pieces, Computation
error, modulus out of range)."""
import ctypes
import glob
import os

import pytest

import ap26_b200 as A
from conftest import GOLDEN, GOLDEN_KS, golden_sol, ref_raw

pytestmark = pytest.mark.gpu

BASES = (2, 3, 5, 7, 11, 13, 17, 19, 23)
P23 = A.PRIM23
SPSP2 = [2 ** p - 1 for p in (11, 23, 29, 37, 41, 43, 47, 53, 59)] + [2 ** 32 + 1]
PSP9 = 3825123056546413051      # composite, strong probable prime to all nine bases


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


def oracle_report(oracle, reports, h0=0):
    """Sequential ao_report over reports: (ok, hash, SOL lines)."""
    h = ctypes.c_int(h0)
    lines = []
    for k, K, first in reports:
        buf = ctypes.create_string_buffer(1 << 12)
        rc = oracle.ao_report(ctypes.byref(h), k, K, ctypes.c_int64(first), buf, len(buf))
        if rc < 0:
            return False, None, None
        lines += buf.value.decode().splitlines()
    return True, h.value, lines


def report_vectors():
    """The reference's own ReportSolution on single reports
    (tests/golden/make_report_vectors.py)."""
    out = []
    with open(os.path.join(GOLDEN, "report_vectors.txt")) as f:
        for ln in f:
            if ln.startswith("#"):
                continue
            k, K, first, h0, st, h, sols = ln.split()
            sl = [] if sols == "-" else [tuple(map(int, x.split(":"))) for x in sols.split(",")]
            out.append(((int(k), int(K), int(first)), int(h0), st, None if h == "-" else int(h), sl))
    return out


def test_sprp_bases_match_reference_vectors(ctx):
    """Every (N, a) verdict of the reference's strong_prp in the fixture,
    the nine validation bases included."""
    Ns, As, Vs = [], [], []
    with open(os.path.join(GOLDEN, "sprp_vectors.txt")) as f:
        for ln in f:
            if ln.startswith("#"):
                continue
            N, a, v = map(int, ln.split())
            if N % 2 == 1 and a < N and 2 <= a <= 31:
                Ns.append(N)
                As.append(a)
                Vs.append(v)
    assert len(set(As)) == 9 and len(Ns) > 1500
    got, _ = ctx.sprp_bases(Ns, As)
    assert got.tolist() == Vs


def test_sprp_bases_pseudoprimes(ctx):
    Ns, As, exp = [], [], []
    for n in SPSP2 + [PSP9]:
        for a in BASES:
            Ns.append(n)
            As.append(a)
            exp.append(int(sprp(a, n)))
    got, _ = ctx.sprp_bases(Ns, As)
    assert got.tolist() == exp
    with pytest.raises(A.AP26Error):
        ctx.sprp_bases([101], [1])


def test_report_matches_reference_vectors(ctx):
    """Status, hash and solutions of every vector equal the reference's."""
    vec = report_vectors()
    assert len(vec) >= 100 and sum(v[2] == "exit" for v in vec) >= 4
    for rep, h0, st, h, sols in vec:
        rc, fin, hh = ctx.report_batch([rep], result_hash=h0)
        if st == "exit":
            assert rc in (A.E_INVALID, A.E_DOMAIN) and fin[0].status == rc, rep
            continue
        assert rc == A.OK and fin[0].status == A.OK, rep
        assert hh == h, rep
        assert fin[0].sols() == sols, rep


def test_report_vectors_in_one_batch(ctx):
    """All completing vectors in one launch: per-report results do not
    depend on the batch, and the summed hash wraps as the reference's."""
    vec = [v for v in report_vectors() if v[2] == "ok"]
    rc, fin, h = ctx.report_batch([v[0] for v in vec], result_hash=0)
    assert rc == A.OK
    for (rep, h0, _, hv, sols), f in zip(vec, fin):
        assert f.sols() == sols, rep
    f = fin[[v[0] for v in vec].index((1, 1, 2047))]   # two empty pieces after the split
    assert f.hash_add == 2047 % 1000 + 1 + 2047 % 1000 + ((2047 + P23) % 1000)
    adds = sum(f.hash_add for f in fin)
    assert h == (adds - 1) % 2000000000 + 1


def test_report_contract_errors(ctx):
    for bad in [(1, 5, 23), (-1, 5, 101), (1, 0, 101), (1, 400_000_001, 101)]:
        rc, fin, _ = ctx.report_batch([bad])
        assert rc == A.E_ARG and fin[0].status == A.E_ARG
    rc, fin, h = ctx.report_batch([], result_hash=5)
    assert rc == A.OK and fin == [] and h == 5


def test_report_recorded_reference_reports(ctx, oracle):
    """Raw reports of every recorded K: hash and SOL lines equal the oracle's
    ReportSolution over them, and the golden SOL files."""
    allreps = []
    for path in sorted(glob.glob(os.path.join(GOLDEN, "ref_raw", "shift*", "*.txt"))):
        K = int(os.path.basename(path)[:-4])
        reps = ref_raw(K, int(os.path.basename(os.path.dirname(path))[5:]))
        allreps += reps
        ok, h_o, lines_o = oracle_report(oracle, reps)
        rc, fin, h = ctx.report_batch(reps, result_hash=0)
        assert ok and rc == A.OK and h == h_o, K
        lines = [f"{ln} {r[1]} {fi}" for r, f in zip(reps, fin) for ln, fi in f.sols()]
        assert lines == lines_o, K
        if K in GOLDEN_KS and "shift0" in path:
            assert "".join(l + "\n" for l in lines) + A.hash_hex(K, K, h) + "\n" == golden_sol(K)
    ok, h_o, _ = oracle_report(oracle, allreps)
    rc, _, h = ctx.report_batch(allreps, result_hash=0)
    assert rc == A.OK and h == h_o


@pytest.mark.parametrize("K", GOLDEN_KS)
def test_search_k_sol_matches_golden(ctx, K):
    h, sols, st = ctx.search_k_sol(K, 0, result_hash=0)
    text = "".join(f"{a} {b} {c}\n" for a, b, c in sols) + A.hash_hex(K, K, h) + "\n"
    assert text == golden_sol(K)
    assert st.error_flags == 0


def test_search_k_sol_continues_hash(ctx):
    """A K in the middle of a workunit: the hash carried in advances exactly as
    the host ReportSolution over the raw reports advances it."""
    K = 43241056
    aps, _ = ctx.search_k(K, 0)
    r = A.Reporter(result_hash=1999999500)
    r.report_all(aps)
    h, sols, _ = ctx.search_k_sol(K, 0, result_hash=1999999500)
    assert h == r.hash.value
    assert [f"{a} {b} {c}" for a, b, c in sols] == r.sol


def ref_states():
    """Checkpoints the reference CPU build wrote while searching the golden K
    (tests/golden/make_ref_states.py): {K: {ITER: result_hash}}, and the
    final hash of each K (the state with K + 1, ITER 0)."""
    mid, final = {}, {}
    with open(os.path.join(GOLDEN, "ref_states.txt")) as f:
        for ln in f:
            if ln.startswith("#"):
                continue
            kmin, kmax, shift, K, it, h = map(int, ln.split())
            if K == kmax + 1:
                final[kmin] = h
            elif it:
                mid.setdefault(K, {})[it] = h
    return mid, final


@pytest.mark.parametrize("K", GOLDEN_KS)
def test_search_k_sol_continues_reference_mid_k_checkpoints(ctx, K):
    """From the reference's checkpoint at ITER 4 and 8 (hash of shift words
    0..ITER-1), the rest of the K ends at the reference's final hash; its
    solutions are the tail of the whole-K solutions."""
    mid, final = ref_states()
    assert sorted(mid[K]) == [4, 8]
    h_all, sols_all, _ = ctx.search_k_sol(K, 0, result_hash=0)
    assert h_all == final[K]
    for it, h0 in mid[K].items():
        h, sols, st = ctx.search_k_sol(K, 0, result_hash=h0, iter=it)
        assert h == final[K], (K, it)
        assert sols == sols_all[len(sols_all) - len(sols):], (K, it)
    with pytest.raises(A.AP26Error):
        ctx.search_k_sol(K, 0, iter=10)


@pytest.mark.parametrize("K", GOLDEN_KS)
def test_search_k_sol_words_gives_the_reference_pass_hashes(ctx, K):
    """Per-word hash sums kept on the device: the hash after shift words 0-3
    and 0-7 equals the result_hash of the reference CPU build's ITER 4 and 8
    checkpoints (tests/golden/ref_states.txt), the last one the final hash;
    SOL lines come grouped by 4-word pass."""
    st = {}
    with open(os.path.join(GOLDEN, "ref_states.txt")) as f:
        for ln in f:
            if not ln.startswith("#"):
                kmin, kmax, shift, KK, it, h = map(int, ln.split())
                st[(kmin, KK, it)] = h
    h, sols, words, at, _ = ctx.search_k_sol_words(K, 0)
    assert at[3] == st[(K, K, 4)]
    assert at[7] == st[(K, K, 8)]
    assert at[9] == h == st[(K, K + 1, 0)]
    passes = [min(w // 4, 2) for w in words]
    assert passes == sorted(passes)
    text = "".join(f"{a} {b} {c}\n" for a, b, c in sols) + A.hash_hex(K, K, h) + "\n"
    assert text == golden_sol(K)
    # continuing from the ITER 4 state gives the same later words
    h4, _, _, at4, _ = ctx.search_k_sol_words(K, 0, result_hash=st[(K, K, 4)], iter=4)
    assert at4[3] == st[(K, K, 4)] and at4[7] == st[(K, K, 8)] and h4 == h
