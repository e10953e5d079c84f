"""Build libap26.so and the `ap26` command in-tree for sm_100a.

    python ap26_b200/build.py   (run by path: importing the package needs the library)

Outputs (git-ignored, shipped with the working tree):
    ap26_b200/libap26.so   C ABI declared in include/ap26.h
    ap26_b200/bin/ap26     the AP26 KMIN KMAX SHIFT command
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libap26.so")
CLI = os.path.join(HERE, "bin", "ap26")

NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
                  "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include")]


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _newer(out, deps):
    if not os.path.exists(out):
        return False
    t = os.path.getmtime(out)
    return all(os.path.getmtime(d) <= t for d in deps)


def build(force=False, verbose_ptxas=False):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(CLI), exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(ROOT, "include", "ap26.h"))
    objs = []
    cu = os.path.join(CSRC, "ap26_capi.cu")
    o = os.path.join(BUILD, "ap26_capi.o")
    if force or not _newer(o, [cu] + headers):
        extra = ["-Xptxas", "-v"] if verbose_ptxas else []
        _run([NVCC] + NVFLAGS + extra + ["-c", cu, "-o", o])
    objs.append(o)
    c = os.path.join(CSRC, "ap26_host.c")
    o = os.path.join(BUILD, "ap26_host.o")
    if force or not _newer(o, [c] + headers):
        _run(["gcc", "-O2", "-fPIC", "-Wall", "-c", c, "-o", o])
    objs.append(o)
    # outputs are written under a temporary name and renamed, so a reader
    # never sees a half-written library or command
    if force or not _newer(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB + ".tmp"] + objs)
        os.replace(LIB + ".tmp", LIB)
    cli = os.path.join(CSRC, "ap26_cli.c")
    if force or not _newer(CLI, [cli, LIB]):
        _run(["gcc", "-O2", "-Wall", "-o", CLI + ".tmp", cli, "-I", os.path.join(ROOT, "include"),
              "-L", HERE, "-lap26", "-Wl,-rpath,$ORIGIN/.."])
        os.replace(CLI + ".tmp", CLI)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose_ptxas="-v" in sys.argv)
