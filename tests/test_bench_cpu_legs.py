"""bench.py's CPU legs without a GPU: the reference baseline samples every
pass of Search_avx2 and combines them into K/s, and the AVX-512 companion
runs a sized slice.  Short samples (one progress tick, one second)."""
import os

import pytest

import bench

REF = os.path.join(bench.ROOT, "oracle", "_ref", "ref_harness")


@pytest.mark.skipif(not os.access(REF, os.X_OK), reason="reference build absent")
def test_reference_sample_covers_every_pass():
    ks = [43241056, 43241061, 43241062]
    kps, wall, n = bench.ref_sample(ks, 1)
    assert n == 3
    # one K of the reference takes minutes per core: K/s on 3 cores is small
    # but positive
    assert 0 < kps < 1
    assert wall > 0


@pytest.mark.skipif(not os.access(REF, os.X_OK), reason="reference build absent")
def test_reference_sample_line_format():
    import subprocess
    out = subprocess.run([REF, "sample", "43241056", "0", "1", "avx2", "8"],
                         capture_output=True, text=True, check=True).stdout
    f = [ln for ln in out.splitlines() if ln.startswith("SAMPLE")][0].split()
    # SAMPLE K n43_done total seconds isa ITER setup_seconds tick_seconds
    assert f[1] == "43241056" and f[5] == "avx2" and f[6] == "8"
    assert int(f[2]) > 0 and float(f[8]) > 0 and float(f[7]) >= 0


def test_avx512_companion_sized_sample():
    import ctypes
    L = ctypes.CDLL(os.path.join(bench.ROOT, "oracle", "liboracle.so"))
    if not L.a5_supported():
        pytest.skip("CPU without AVX-512 VBMI2")
    c = bench.avx512_companion(43241056, seconds=1.0)
    assert c["kind"] == "port" and c["cores"] == (os.cpu_count() or 1)
    assert 0 < c["value"] < 1
