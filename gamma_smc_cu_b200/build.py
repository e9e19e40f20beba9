"""Build the in-tree CUDA library ``gamma_smc_cu_b200/lib/libgsmc_b200.so``.

nvcc cross-compiles for sm_100a (no GPU needed).  The host table builder is
compiled by g++ with -ffp-contract=off so its FP32 arithmetic matches the
reference's table builder bit for bit.

    python -m gamma_smc_cu_b200.build [--force]
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
OBJDIR = os.path.join(HERE, "_build")
LIB = os.path.join(LIBDIR, "libgsmc_b200.so")

CUDA_SOURCES = ["scan.cu", "capi.cu", "hostcopy.cu", "exec.cu", "fwd.cu", "flowgen.cu", "uncached.cu",
                "noalloc.cu", "tables_gpu.cu"]
CXX_SOURCES = ["tables.cpp"]
HEADERS = ["scan.h", "scan_device.cuh", "tables.h", "hostcopy.h", "ctx_view.h", "fwd.h", "flowgen.h", "uncached.h",
           "windows.h", "tables_gpu.h", "planner.h"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
              "--expt-relaxed-constexpr", "-Xptxas", "-v"] + ARCH
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-ffp-contract=off", "-pthread"]


def _nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else (shutil.which("nvcc") or "nvcc")


def _cxx():
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(OBJDIR, exist_ok=True)
    inc = ["-I", CSRC, "-I", os.path.join(REPO, "include")]
    headers = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(REPO, "include", "gsmc_b200.h")]
    objs = []
    for src in CUDA_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJDIR, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            cmd = [_nvcc()] + NVCC_FLAGS + inc + ["-c", s, "-o", o]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if verbose or r.returncode:
                sys.stderr.write(r.stdout + r.stderr)
            if r.returncode:
                raise RuntimeError(f"nvcc failed on {src}")
    for src in CXX_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJDIR, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            cmd = [_cxx()] + CXX_FLAGS + inc + ["-c", s, "-o", o]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode:
                sys.stderr.write(r.stdout + r.stderr)
                raise RuntimeError(f"g++ failed on {src}")
    if force or _stale(LIB, objs):
        cmd = [_nvcc(), "-shared"] + ARCH + objs + ["-o", LIB, "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("nvcc link failed")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
