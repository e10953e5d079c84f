"""CPU tests of libap26.so: it loads, exports every symbol include/ap26.h
declares, refuses to run without a GPU (no CPU fallback), and its host
services reproduce the reference's SOL files, hash and state files."""
import ctypes
import os
import re
import subprocess

import pytest

from conftest import GOLDEN_KS, ROOT, golden_sol, ref_raw

import ap26_b200 as A


def header_symbols():
    with open(os.path.join(ROOT, "include", "ap26.h")) as f:
        text = f.read()
    return sorted(set(re.findall(r"\b(ap26_[a-z0-9_]+)\s*\(", text)))


def test_exports_every_declared_symbol():
    syms = header_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(A.lib, s), f"libap26.so does not export {s}"
    assert set(syms) == set(A.EXPORTS)


def test_version_and_strerror():
    assert A.lib.ap26_version() >= 10000
    for code in range(-9, 1):
        assert A.lib.ap26_strerror(code)


def test_will_search_matches_reference_rule():
    # AP26.cpp:649-653: K divisible by any of 29..59 is skipped
    for K in range(1, 5000):
        exp = all(K % p for p in (29, 31, 37, 41, 43, 47, 53, 59))
        assert A.will_search(K) == exp


@pytest.mark.parametrize("K", GOLDEN_KS)
def test_report_and_hash_reproduce_golden_sol(K):
    """Reference raw reports -> ReportSolution/write_hash restatement ->
    the reference's own golden SOL file, byte for byte."""
    r = A.Reporter()
    r.report_all(ref_raw(K))
    assert r.sol_file(K, K) == golden_sol(K)


def test_hash_hex_edge_cases():
    assert A.hash_hex(0, 0, 0) == "0000000000000000"
    assert A.hash_hex(366384, 366384, 87376) == "000B2E6000015550"
    # KMIN+KMAX above MAXINTV (but inside int) wraps by 2e9 (AP26.cpp:310-312)
    assert A.hash_hex(1_000_000_000, 1_100_000_000, 1) == \
        "%08X%08X" % (2_100_000_000 - 2_000_000_000, 1)


def test_report_rejects_non_base2_ap():
    r = A.Reporter()
    with pytest.raises(A.AP26Error) as e:
        r.report(12, 366384, 6171054912832631 + 1)   # even first term: not an AP of primes
    assert e.value.code == A.E_INVALID


def test_report_splits_non_solutions():
    """A base-2 AP that fails the 9-base check is split (AP26.cpp:565-582);
    the hash counts the raw AP and every piece, including empty ones."""
    import ctypes
    # the golden length-25 AP extended by one composite-free term is not a
    # valid 26-AP: its last term fails base 2, so report a shorter raw AP.
    r = A.Reporter()
    r.report(25, 366384, 6171054912832631)
    assert r.sol == ["25 366384 6171054912832631"]
    assert r.hash.value == 631 + 25


def test_state_files_roundtrip(tmp_path):
    import ctypes
    d = str(tmp_path).encode()
    wa = ctypes.c_int(1)
    assert A.lib.ap26_write_state(d, 10, 20, 0, 12, 0, 555, 1.5, ctypes.byref(wa)) == 0
    assert wa.value == 0  # next write goes to B
    assert A.lib.ap26_write_state(d, 10, 20, 0, 13, 0, 777, 2.0, ctypes.byref(wa)) == 0
    assert open(tmp_path / "AP26-state.a.txt").read() == "10 20 0 12 0 555 1.500000\n"
    assert open(tmp_path / "AP26-state.b.txt").read() == "10 20 0 13 0 777 2.000000\n"
    K, IT, h, tr, nxt = (ctypes.c_int(), ctypes.c_int(), ctypes.c_int32(), ctypes.c_double(),
                         ctypes.c_int())
    ok = A.lib.ap26_read_state(d, 10, 20, 0, ctypes.byref(K), ctypes.byref(IT), ctypes.byref(h),
                               ctypes.byref(tr), ctypes.byref(nxt))
    assert ok == 1 and K.value == 13 and h.value == 777 and nxt.value == 1
    # mismatched workunit parameters are ignored (AP26.cpp:420)
    assert A.lib.ap26_read_state(d, 10, 21, 0, ctypes.byref(K), ctypes.byref(IT),
                                 ctypes.byref(h), ctypes.byref(tr), ctypes.byref(nxt)) == 0
    # a corrupt newer file falls back to the other one
    (tmp_path / "AP26-state.b.txt").write_text("garbage\n")
    ok = A.lib.ap26_read_state(d, 10, 20, 0, ctypes.byref(K), ctypes.byref(IT), ctypes.byref(h),
                               ctypes.byref(tr), ctypes.byref(nxt))
    assert ok == 1 and K.value == 12 and h.value == 555 and nxt.value == 0
    # truncated files on both sides: fresh start
    (tmp_path / "AP26-state.a.txt").write_text("10 20 0")
    assert A.lib.ap26_read_state(d, 10, 20, 0, ctypes.byref(K), ctypes.byref(IT),
                                 ctypes.byref(h), ctypes.byref(tr), ctypes.byref(nxt)) == 0


def test_context_without_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(A.AP26Error) as e:
        A.Context(0)
    assert e.value.code in (A.E_NODEV, A.E_CUDA)


def test_cli_without_gpu_exits_nonzero(tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    p = subprocess.run([A.CLI_PATH, "366384", "366384", "0"], cwd=tmp_path, capture_output=True,
                       text=True)
    assert p.returncode != 0
    assert not (tmp_path / "SOL-AP26.txt").exists()


@pytest.mark.parametrize("cname,pyname", [
    ("ap26_opts", "Opts"), ("ap26_ap", "AP"), ("ap26_stats", "Stats"), ("ap26_item", "Item"),
    ("ap26_item_result", "ItemResult"), ("ap26_final", "Final"), ("ap26_sol", "Sol")])
def test_ctypes_structures_match_the_header(tmp_path, cname, pyname):
    """Every ctypes mirror has the C struct's size and field offsets, as
    include/ap26.h declares them (compiled here with the host C compiler)."""
    import shutil
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no host C compiler")
    py = getattr(A, pyname)
    fields = [f for f, _ in py._fields_]
    src = tmp_path / "layout.c"
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "ap26.h"', "int main(void) {",
             f'  printf("%zu\\n", sizeof({cname}));']
    lines += [f'  printf("%zu\\n", offsetof({cname}, {f}));' for f in fields]
    lines += ["  return 0;", "}"]
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    subprocess.run([cc, "-std=c11", "-I", inc, str(src), "-o", str(exe)], check=True)
    out = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True,
                                          text=True).stdout.split()]
    assert out[0] == ctypes.sizeof(py), (cname, out[0], ctypes.sizeof(py))
    assert out[1:] == [getattr(py, f).offset for f in fields], cname
