"""Builds the host emulator (tests/native/_build/libbtemu.so): test-only."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "_build", "libbtemu.so")


def build() -> str:
    src = os.path.join(HERE, "emu.cpp")
    deps = [src] + [os.path.join(ROOT, "beamtrace2007_b200", "csrc", f) for f in ("beam_math.cuh", "engine_core.cuh")]
    if os.path.exists(OUT) and all(os.path.getmtime(d) <= os.path.getmtime(OUT) for d in deps):
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    cuda_inc = "/usr/local/cuda/include"
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-fvisibility=hidden",
           "-I" + os.path.join(ROOT, "include"), "-I" + os.path.join(ROOT, "beamtrace2007_b200", "csrc"),
           "-I" + cuda_inc, "-o", OUT, src]
    subprocess.run(cmd, check=True)
    return OUT
