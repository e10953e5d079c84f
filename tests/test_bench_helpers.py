"""CPU tests of bench.py's parity helpers: a parity key reports ok only
when it checked something and every checked item equals the reference's
recorded reports and their ReportSolution hash (tests/golden/ref_raw)."""
import sys

from conftest import ROOT, ref_raw

import ap26_b200 as A

sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _hash(reps):
    r = A.Reporter()
    r.report_all(reps)
    return r.hash.value


def test_item_parity_ok_only_for_matching_checked_items():
    K = 43241061                                   # a recorded reference fixture
    reps = [(k, KK, f, 0) for k, KK, f in ref_raw(K)]
    item = [(1, K, K, 0)]
    ok = bench.item_parity(A, item, [reps], [_hash(ref_raw(K))])
    assert ok["ok"] and ok["items_checked_vs_reference"] == 1 and ok["all_items_checked"]
    # one report dropped: the reports and the hash differ
    bad = bench.item_parity(A, item, [reps[:-1]], [_hash(ref_raw(K)[:-1])])
    assert not bad["ok"] and bad["mismatched"] == [1]
    # the right reports with a wrong hash
    bad = bench.item_parity(A, item, [reps], [_hash(ref_raw(K)) + 1])
    assert not bad["ok"]


def test_item_parity_with_nothing_checked_is_not_ok():
    K = 27872096 + 10 ** 6                         # no fixture recorded
    assert bench.ref_fixture(K, 640) is None
    res = bench.item_parity(A, [(5, K, K, 640)], [[]], [0])
    assert res["items_checked_vs_reference"] == 0 and not res["ok"]


def test_parity_check_needs_a_checked_k():
    K = 43241061
    seen = {K: [tuple(r) for r in ref_raw(K)]}
    assert bench.parity_check(seen, K)["ok"]
    seen[K] = seen[K][1:]
    assert not bench.parity_check(seen, K)["ok"]
    assert not bench.parity_check({}, K)["ok"]


def test_reference_counts_cover_the_sieve_pair_prefix():
    """Every searchable K of the sieve pair's first 64 has a reference count."""
    pinned = bench.ref_counts()
    ks = [k for k in bench.sieve_pair_ks() if bench.will_search(k)]
    assert len(ks) == bench.SIEVE_PAIR_PINNED
    assert all((k, bench.SIEVE_PAIR_SHIFT) in pinned for k in ks)
