"""Shared fixtures.

Markers:
  gpu   needs a CUDA device (run with -m gpu on a B200)
"""
import ctypes
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _oracle_lib():
    path = os.path.join(ROOT, "oracle", "liboracle.so")
    srcs = [os.path.join(ROOT, "oracle", f) for f in ("ap26_oracle.c", "ap26_avx512.c")]
    if not os.path.exists(path) or any(os.path.getmtime(path) < os.path.getmtime(s)
                                       for s in srcs):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "liboracle.so"],
                       check=True)
    L = ctypes.CDLL(path)
    L.ao_search.restype = ctypes.c_int64
    L.ao_sieve.restype = ctypes.c_int64
    L.ao_n59.restype = ctypes.c_int64
    L.ao_avx2_order_key.restype = ctypes.c_uint64
    L.ao_avx2_order_key.argtypes = [ctypes.c_uint64]
    L.a5_sieve.restype = ctypes.c_int64
    L.a5_search.restype = ctypes.c_int64
    return L


@pytest.fixture(scope="session")
def oracle():
    """The CPU oracle (oracle/ap26_oracle.c), the checker for every test."""
    return _oracle_lib()


@pytest.fixture(scope="session")
def ctx():
    """One libap26 device context for the whole GPU session."""
    import ap26_b200 as A
    c = A.Context(0)
    yield c
    c.close()


def ref_raw(K, shift=0):
    """Raw reports recorded from the reference's own Search_avx2."""
    path = os.path.join(GOLDEN, "ref_raw", f"shift{shift}", f"{K}.txt")
    out = []
    with open(path) as f:
        for ln in f:
            if ln.startswith("#"):
                continue
            k, KK, first = map(int, ln.split())
            out.append((k, KK, first))
    return out


def golden_sol(K):
    with open(os.path.join(GOLDEN, f"TEST-{K}.txt")) as f:
        return f.read()


GOLDEN_KS = (366384, 44121555, 47715109)
