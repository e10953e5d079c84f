"""Serving with continuous batching (ap26_serve_*), on the GPU.

A unit is every searchable K of an item.  Units are admitted while the
serving pool has device memory for their sieve tables; ap26_serve_step never
blocks, keeping two slices of K-jobs queued on the device; each unit keeps its
running ReportSolution hash and its checkpoint (the reference's state-file
fields, src/common/AP26.cpp:360-390) on the device.  Checked here: units
submitted while slices run are admitted without waiting for the device and
join the next slice; every unit's reports and result hash equal the
reference's own (tests/golden/ref_raw, recorded from the reference's
Search_avx2 and folded through the host ReportSolution); a unit's device
checkpoint round-trips through ap26_write_state / ap26_read_state and a unit
resumed from it ends with the uninterrupted unit's hash; admission refuses
units whose tables do not fit.
"""
import ctypes
import time

import pytest

from conftest import ref_raw

import ap26_b200 as A

pytestmark = pytest.mark.gpu


def _drain(c, limit_s=600):
    """Steps the service until every admitted unit is finished; returns the
    polled results {id: (result, reports)}."""
    out = {}
    t0 = time.time()
    while True:
        active = c.serve_step()
        while True:
            r = c.serve_poll()
            if r is None:
                break
            out[r[0].id] = r
        if active == 0:
            return out
        assert time.time() - t0 < limit_s
        c.serve_wait(1.0)


def _expected(units):
    """Reports and result_hash of each unit from the reference's raw reports."""
    exp = {}
    for uid, kmin, kmax, shift in units:
        reps = []
        for K in range(kmin, kmax + 1):
            if A.will_search(K):
                reps += ref_raw(K, shift)
        r = A.Reporter()
        r.report_all(reps)
        exp[uid] = (reps, r.hash.value)
    return exp


# units whose every searchable K has a recorded reference fixture
FIXTURE_UNITS = [(11, 43241056, 43241062, 0), (12, 17973973, 17973973, 640),
                 (13, 43241064, 43241068, 0), (14, 28096782, 28096782, 1280),
                 (15, 7928262, 7928262, 15360)]


def test_serving_units_equal_reference_reports_and_hash():
    exp = _expected(FIXTURE_UNITS)
    with A.Context(0) as c:
        for u in FIXTURE_UNITS:
            assert c.serve_submit(*u) == 0
        got = _drain(c)
    assert sorted(got) == sorted(exp)
    for uid, (res, aps) in got.items():
        reps, h = exp[uid]
        assert res.status == 0
        assert [(k, K, f) for k, K, f, _ in aps] == reps, uid
        assert res.result_hash == h, uid
        assert res.ks_searched == sum(A.will_search(K) for K in range(
            *[(a, b + 1) for i, a, b, _ in FIXTURE_UNITS if i == uid][0]))


def test_submit_while_slices_run_does_not_wait_for_the_device():
    """Two slices are queued by the first step (about 3 s of device work);
    a unit submitted then is admitted at once (its tables are enqueued, not
    waited for), is not in the queued slices, and joins a later one."""
    first = (21, 3000017, 3000029, 0)            # 10 searchable K
    late = (22, 43241061, 43241061, 0)
    with A.Context(0) as c:
        assert c.serve_submit(*first) == 0
        t0 = time.perf_counter()
        active = c.serve_step()
        t_step = time.perf_counter() - t0
        assert active == 1
        assert c.serve_wait(0.0) is False        # a slice is still on the device
        t0 = time.perf_counter()
        assert c.serve_submit(*late) == 0
        t_submit = time.perf_counter() - t0
        t0 = time.perf_counter()
        c.serve_step()
        t_step2 = time.perf_counter() - t0
        assert c.serve_wait(0.0) is False        # ... and still is: nothing waited for it
        # no call waited for a slice (a slice of 4 K takes about 1.5 s)
        assert t_step < 0.25 and t_submit < 0.25 and t_step2 < 0.25, (t_step, t_submit, t_step2)
        got = _drain(c)
    reps = ref_raw(43241061)
    r = A.Reporter()
    r.report_all(reps)
    res, aps = got[22]
    assert [(k, K, f) for k, K, f, _ in aps] == reps
    assert res.result_hash == r.hash.value
    assert got[21][0].ks_searched == 10 and got[21][0].status == 0


def test_device_checkpoint_roundtrips_through_state_files(tmp_path):
    """A unit's device checkpoint after some slices, written with
    ap26_write_state and read back with ap26_read_state, resumes in a fresh
    context to the uninterrupted unit's reports (the remaining ones) and
    result hash; the checkpoint fields are the reference's state fields."""
    unit = (31, 43241056, 43241069, 0)    # 9 searchable K, all with fixtures
    exp_reps, exp_hash = _expected([unit])[31]
    with A.Context(0) as c:
        assert c.serve_submit(*unit) == 0
        kmin, kmax, shift, K, IT, h = c.serve_checkpoint(31)
        assert (kmin, kmax, shift, K, IT, h) == (unit[1], unit[2], unit[3], unit[1], 0, 0)
        # run until the first slice has come back, then take the checkpoint
        c.serve_step()
        assert c.serve_wait(600.0)
        c.serve_step()
        kmin, kmax, shift, K, IT, h = c.serve_checkpoint(31)
    assert (kmin, kmax, shift, IT) == (unit[1], unit[2], unit[3], 0)
    assert unit[1] < K <= unit[2]
    # the state the checkpoint names: hash of every report of K' < K
    done = [x for x in range(unit[1], K) if A.will_search(x)]
    r = A.Reporter()
    for x in done:
        r.report_all(ref_raw(x))
    assert h == r.hash.value
    d = str(tmp_path).encode()
    wa = ctypes.c_int(1)
    assert A.lib.ap26_write_state(d, kmin, kmax, shift, K, IT, h, 0.0, ctypes.byref(wa)) == 0
    K2, IT2, h2, tr, nxt = (ctypes.c_int(), ctypes.c_int(), ctypes.c_int32(), ctypes.c_double(),
                            ctypes.c_int())
    assert A.lib.ap26_read_state(d, kmin, kmax, shift, ctypes.byref(K2), ctypes.byref(IT2),
                                 ctypes.byref(h2), ctypes.byref(tr), ctypes.byref(nxt)) == 1
    assert (K2.value, IT2.value, h2.value) == (K, IT, h)
    with A.Context(0) as c:
        assert c.serve_submit_from(32, kmin, kmax, shift, K2.value, IT2.value, h2.value) == 0
        got = _drain(c)
    res, aps = got[32]
    tail = [t for x in range(K, unit[2] + 1) if A.will_search(x) for t in ref_raw(x)]
    assert [(k, KK, f) for k, KK, f, _ in aps] == tail
    assert tail == exp_reps[len(exp_reps) - len(tail):]
    assert res.result_hash == exp_hash


def test_unit_resumed_mid_k_from_a_reference_cpu_checkpoint():
    """ap26_serve_submit_from with a state the reference CPU build writes
    before its second 4-word pass (K=366384, ITER 4, tests/golden/ref_states.txt)
    ends at the reference's final hash."""
    with A.Context(0) as c:
        assert c.serve_submit_from(41, 366384, 366384, 0, 366384, 4, 48373) == 0
        got = _drain(c)
        assert c.serve_submit_from(42, 366384, 366384, 0, 366384, 8, 72858) == 0
        got.update(_drain(c))
    assert got[41][0].result_hash == 87376
    assert got[42][0].result_hash == 87376


def test_admission_by_device_memory():
    """The pool of tables is sized from mem_budget at the first admission:
    each admitted unit holds its K's tables (the same bytes per K), a unit
    whose tables do not fit is refused (AP26_E_NOMEM), and a unit's bytes
    return when it finishes."""
    with A.Context(0, mem_budget=24 << 20) as c:
        assert c.serve_submit(51, 1_000_003, 1_000_003, 0) == 0        # 1 searchable K
        held1, budget = c.serve_memory()
        assert budget <= 24 << 20
        assert c.serve_submit(52, 2_000_003, 2_000_004, 0) == 0        # 2 searchable K
        held2, _ = c.serve_memory()
        per_k = (held2 - held1) // 2
        assert per_k > 10_000 and held2 - held1 == 2 * per_k
        room = (budget - held2) // per_k
        assert c.serve_submit(53, 1_000_003, 1_000_003 + 3 * room, 0) == A.E_NOMEM
        _drain(c)
        held3, _ = c.serve_memory()
        assert held3 == held1 - per_k


def test_densest_k_runs_and_serves_without_overflow():
    """K = 61*67*71*73 = 21182921 is the densest searchable K below 4e8: the
    four smallest sieve primes divide K*23#, so each bans one residue
    instead of 24 and about 5.4 times the usual candidates survive.  The
    synchronous search redoes an overflowing chunk in smaller ones (here a
    2^24-entry ring forces it); serving slices size their chunks for this
    density.  Both give the reference's reports."""
    K = 21182921
    ref = ref_raw(K)
    with A.Context(0, cand_ring_log2=24) as c:
        aps, st = c.search_k(K, 0)
        assert st.error_flags & 1                 # redone in smaller chunks
    assert [(k, KK, f) for k, KK, f, _ in aps] == ref
    assert st.candidates > 5 * 36_000_000
    with A.Context(0) as c:
        assert c.serve_submit(61, K, K, 0) == 0
        got = _drain(c)
    res, saps = got[61]
    assert res.status == 0
    assert [(k, KK, f) for k, KK, f, _ in saps] == ref
    assert res.candidates == st.candidates
    r = A.Reporter()
    r.report_all(ref)
    assert res.result_hash == r.hash.value
