"""The ap26 command (the reference's CLI contract, src/common/AP26.cpp:660-1041)
on the GPU: golden SOL file, A/B checkpoint files, resume after a stop
between K, and the batched form writing the same output."""
import os
import subprocess

import pytest

from conftest import golden_sol, ref_raw

import ap26_b200 as A

pytestmark = pytest.mark.gpu


def run_cli(cwd, *args):
    p = subprocess.run([A.CLI_PATH] + [str(a) for a in args], cwd=cwd, capture_output=True,
                       text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    return p


def test_cli_reproduces_golden_sol_and_final_state(tmp_path):
    run_cli(tmp_path, 366384, 366384, 0)
    assert (tmp_path / "SOL-AP26.txt").read_text() == golden_sol(366384)
    # the states written alternate A/B as the reference's: before the K
    # (A), after its 4-word passes at ITER 4 (B) and ITER 8 (A), and the
    # final one with K = KMAX+1 (B); the files keep the last two
    # (tests/golden/ref_states.txt)
    a = (tmp_path / "AP26-state.a.txt").read_text().split()
    b = (tmp_path / "AP26-state.b.txt").read_text().split()
    assert a[:6] == ["366384", "366384", "0", "366384", "8", "72858"]
    assert b[:6] == ["366384", "366384", "0", "366385", "0", "87376"]


def test_cli_resume_equals_uninterrupted_run(tmp_path):
    kmin, kmax = 366384, 366386        # 366385 is searchable; 366386 = 29 * 12634 is skipped
    full = tmp_path / "full"
    full.mkdir()
    run_cli(full, kmin, kmax, 0)
    expected = (full / "SOL-AP26.txt").read_text()
    # a run stopped after its first K: the checkpoint written before K=366385
    # holds K=366385 and the hash of K=366384 (87376), as the reference writes
    part = tmp_path / "resumed"
    part.mkdir()
    r = A.Reporter()
    r.report_all(ref_raw(366384))
    (part / "AP26-state.a.txt").write_text(f"{kmin} {kmax} 0 366385 0 {r.hash.value} 0.000000\n")
    (part / "SOL-AP26.txt").write_text("".join(l + "\n" for l in r.sol))
    p = run_cli(part, kmin, kmax, 0)
    assert "Resuming" in p.stdout
    assert (part / "SOL-AP26.txt").read_text() == expected


def test_cli_batched_form_writes_same_output(tmp_path):
    a = tmp_path / "plain"
    b = tmp_path / "batched"
    a.mkdir()
    b.mkdir()
    run_cli(a, 1000037, 1000041, 640)
    run_cli(b, 1000037, 1000041, 640, "-batch", 3)
    assert (a / "SOL-AP26.txt").read_text() == (b / "SOL-AP26.txt").read_text()


def test_cli_continues_reference_mid_k_checkpoint(tmp_path):
    """A state written by the reference CPU build before its second 4-word
    pass (K=366384, ITER=4, hash 48373; tests/golden/ref_states.txt), with the
    SOL lines it had written by then: the command continues the K at shift
    word 4 and ends with the golden SOL file."""
    mid = {}
    with open(os.path.join(os.path.dirname(__file__), "golden", "ref_states.txt")) as f:
        for ln in f:
            if not ln.startswith("#"):
                kmin, kmax, shift, K, it, h = map(int, ln.split())
                mid[(K, it)] = h
    K = 366384
    with A.Context(0) as c:
        _, sols_all, _ = c.search_k_sol(K, 0)
        _, sols_tail, _ = c.search_k_sol(K, 0, result_hash=mid[(K, 4)], iter=4)
    head = sols_all[:len(sols_all) - len(sols_tail)]
    (tmp_path / "AP26-state.a.txt").write_text(f"{K} {K} 0 {K} 4 {mid[(K, 4)]} 0.000000\n")
    (tmp_path / "SOL-AP26.txt").write_text("".join(f"{a} {b} {c}\n" for a, b, c in head))
    p = run_cli(tmp_path, K, K, 0)
    assert "Continuing K 366384 from shift word 4" in p.stderr
    assert (tmp_path / "SOL-AP26.txt").read_text() == golden_sol(K)
    states = [(tmp_path / f).read_text().split()[:6]
              for f in ("AP26-state.a.txt", "AP26-state.b.txt")]
    assert [str(K), str(K), "0", str(K + 1), "0", "87376"] in states



def test_cli_stopped_between_k_resumes_to_same_output(tmp_path):
    """The process ends after each searched K (-stop-after 1: checkpoint of
    the next K written, no hash line) and is started again until done: the
    SOL file equals the uninterrupted run's."""
    kmin, kmax = 366384, 366388          # 366386 = 29 * 12634 is skipped
    full = tmp_path / "full"
    full.mkdir()
    run_cli(full, kmin, kmax, 0)
    part = tmp_path / "stopped"
    part.mkdir()
    runs = 0
    while True:
        p = run_cli(part, kmin, kmax, 0, "-stop-after", 1)
        runs += 1
        if "Workunit complete" in p.stderr:
            break
        assert "Stopped after 1 K" in p.stderr
        assert runs < 10
    assert runs == 4                     # 4 searchable K
    assert (part / "SOL-AP26.txt").read_text() == (full / "SOL-AP26.txt").read_text()


def test_cli_whole_64k_workunit_matches_reference(tmp_path, oracle):
    """The bench's 64-K workunit (KMIN 43241056, SHIFT 0; 51 searchable K)
    through the command in batched mode: SOL lines and hash equal the
    reference's ReportSolution over its own raw reports of every K
    (tests/golden/ref_raw/shift0), in K order."""
    import ctypes
    kmin, kmax = 43241056, 43241056 + 63
    h = ctypes.c_int(0)
    sol = ctypes.create_string_buffer(1 << 16)
    n = 0
    for K in range(kmin, kmax + 1):
        if not A.will_search(K):
            continue
        n += 1
        for k, KK, first in ref_raw(K):
            assert oracle.ao_report(ctypes.byref(h), k, KK, ctypes.c_int64(first), sol,
                                    len(sol)) == 0
    assert n == 51
    hexb = ctypes.create_string_buffer(17)
    oracle.ao_hash_hex(kmin, kmax, h, hexb)
    expected = sol.value.decode() + hexb.value.decode() + "\n"
    run_cli(tmp_path, kmin, kmax, 0, "-batch", 16)
    assert (tmp_path / "SOL-AP26.txt").read_text() == expected


def _ref_states():
    """(K, ITER) -> result_hash of the states the reference CLI wrote while
    searching the golden K (tests/golden/ref_states.txt)."""
    out = {}
    with open(os.path.join(os.path.dirname(__file__), "golden", "ref_states.txt")) as f:
        for ln in f:
            if not ln.startswith("#"):
                kmin, kmax, shift, K, it, h = map(int, ln.split())
                out[(kmin, K, it)] = h
    return out


def _newest_state(d, kmin, kmax, shift):
    import ctypes
    K, IT, h, tr, nxt = (ctypes.c_int(), ctypes.c_int(), ctypes.c_int32(), ctypes.c_double(),
                         ctypes.c_int())
    ok = A.lib.ap26_read_state(str(d).encode(), kmin, kmax, shift, ctypes.byref(K),
                               ctypes.byref(IT), ctypes.byref(h), ctypes.byref(tr),
                               ctypes.byref(nxt))
    assert ok == 1
    return K.value, IT.value, h.value


@pytest.mark.parametrize("K", (366384, 44121555, 47715109))
def test_cli_writes_the_reference_per_pass_states(tmp_path, K):
    """Inside a K the command writes the states the reference CPU build
    writes between its 4-word passes (src/cpu/cpuavx2.cpp:858-861).  Stopped
    right after the ITER 4 state and again after the ITER 8 state, the newest
    state equals the reference's (tests/golden/ref_states.txt), the SOL file
    holds a prefix of the golden lines, and the run resumed from there ends
    with the golden SOL file and the reference's final state."""
    st = _ref_states()
    golden = golden_sol(K).splitlines()
    p = run_cli(tmp_path, K, K, 0, "-stop-at-word", 4)
    assert "Checkpoint: KMIN:%d KMAX:%d SHIFT:0 K:%d ITER:4" % (K, K, K) in p.stdout
    assert _newest_state(tmp_path, K, K, 0) == (K, 4, st[(K, K, 4)])
    sol = (tmp_path / "SOL-AP26.txt")
    part = sol.read_text().splitlines() if sol.exists() else []
    assert part == golden[:len(part)]
    run_cli(tmp_path, K, K, 0, "-stop-at-word", 8)
    assert _newest_state(tmp_path, K, K, 0) == (K, 8, st[(K, K, 8)])
    part2 = sol.read_text().splitlines() if sol.exists() else []
    assert part2 == golden[:len(part2)] and len(part2) >= len(part)
    run_cli(tmp_path, K, K, 0)
    assert sol.read_text() == golden_sol(K)
    assert _newest_state(tmp_path, K, K, 0) == (K + 1, 0, st[(K, K + 1, 0)])
