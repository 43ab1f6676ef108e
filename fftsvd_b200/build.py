"""Build the in-tree shared library fftsvd_b200/libfftsvd_b200.so.

CUDA sources are compiled for sm_100a only (-gencode arch=compute_100a,code=sm_100a);
host-only C++ (the operator setup) is compiled with the host compiler and OpenMP.
Objects are rebuilt when their source or any header is newer.

    python -m fftsvd_b200.build [--force] [--debug]
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libfftsvd_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    cand = [os.environ.get("NVCC", ""), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc") or ""]
    for c in cand:
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _host_cxx() -> str:
    # the environment's CC/CXX may point at a compiler without OpenMP support files
    for c in ("/usr/bin/g++", shutil.which("g++") or ""):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("g++ not found")


def _newest_header() -> float:
    hs = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh"))
    hs.append(os.path.join(ROOT, "include", "fftsvd_b200.h"))
    return max(os.path.getmtime(h) for h in hs if os.path.exists(h))


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"compile failed: {cmd[-1] if cmd else ''}")
    return r


def build(force: bool = False, debug: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    cxx = _host_cxx()
    hdr = _newest_header()
    opt = ["-O0", "-g"] if debug else ["-O3"]
    objs = []
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cu"))):
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(src), hdr):
            cmd = [nvcc, *ARCH, "-lineinfo", *opt, "-std=c++17", "-Xcompiler", "-fPIC,-fopenmp", "--expt-relaxed-constexpr",
                   "-ccbin", cxx, "-I", os.path.join(ROOT, "include"), "-c", src, "-o", obj]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
            r = _run(cmd)
            if verbose:
                sys.stderr.write(r.stderr)
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cpp"))):
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(src), hdr):
            _run([cxx, *opt, "-std=c++17", "-fPIC", "-fopenmp", "-march=x86-64-v3", "-I", os.path.join(ROOT, "include"),
                  "-I", "/usr/local/cuda/include", "-c", src, "-o", obj])
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        _run([nvcc, *ARCH, "-shared", "-ccbin", cxx, "-Xcompiler", "-fopenmp", "-o", LIB, *objs,
              "-lgomp", "-cudart", "static"])
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, debug="--debug" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
