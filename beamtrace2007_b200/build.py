"""Builds libbt_gpu.so in-tree: the sm_100a CUDA engine plus the host-side
scene code, behind the C-ABI of include/bt_gpu.h.

    python -m beamtrace2007_b200.build          # or __graft_entry__.build()

Floating-point flags keep every beam operation IEEE single precision in the
reference's order: -fmad=false (no contraction into FMA), IEEE division and
square root, no flush-to-zero; host code with -ffp-contract=off.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(PKG, "libbt_gpu.so")
OBJ = os.path.join(ROOT, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
              "-Xcompiler", "-fPIC,-ffp-contract=off,-fvisibility=hidden", "--expt-relaxed-constexpr",
              "-I" + INCLUDE, "-I" + CSRC]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fvisibility=hidden", "-I" + INCLUDE]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} {os.path.basename(cmd[-1])}")
    return r.stdout + r.stderr


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(INCLUDE, "bt_gpu.h"))
    objs = []
    log = ""
    for src in sorted(os.listdir(CSRC)):
        path = os.path.join(CSRC, src)
        if src.endswith(".cu"):
            obj = os.path.join(OBJ, src + ".o")
            if force or _stale(obj, [path] + headers):
                extra = ["-Xptxas", "-v"] if ptxas_info else []
                log += _run([nvcc()] + ARCH + NVCC_FLAGS + extra + ["-c", "-o", obj, path])
            objs.append(obj)
        elif src.endswith(".cpp"):
            obj = os.path.join(OBJ, src + ".o")
            if force or _stale(obj, [path] + headers):
                log += _run(["g++"] + CXX_FLAGS + ["-c", "-o", obj, path])
            objs.append(obj)
    if force or _stale(LIB, objs):
        log += _run([nvcc()] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-o", LIB] + objs + ["-lpthread"])
    if verbose and log:
        print(log)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
