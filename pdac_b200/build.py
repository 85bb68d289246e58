"""Build the engine's CUDA library in-tree for sm_100a (B200).

``python -m pdac_b200.build`` (or ``__graft_entry__.build()``) runs nvcc on
``pdac_b200/csrc/engine.cu`` and writes ``pdac_b200/_lib/libpdac_b200.so``.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libpdac_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

# FP64 parity mode: no FMA contraction, so each product and sum rounds as in
# the reference's source order.
FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "--extended-lambda",
    "-fmad=false", "-Xcompiler", "-fPIC", "-shared",
]


def sources():
    return [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC)) if f.endswith((".cu", ".cuh", ".h"))]


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + [os.path.join(HERE, "..", "include", "pdac_gpu.h")]
    return any(os.path.getmtime(s) > t for s in deps)


HOST_SRC = os.path.join(HERE, "host", "pdac_run.cpp")
HOST_BIN = os.path.join(OUT_DIR, "pdac_run")


def build_host(force=False):
    """The compiled time-loop driver (pdac_b200/host/pdac_run.cpp), linked
    against the engine library with the library's directory as its run path."""
    if not force and os.path.exists(HOST_BIN) and os.path.getmtime(HOST_BIN) >= max(
            os.path.getmtime(HOST_SRC), os.path.getmtime(LIB)):
        return HOST_BIN
    cmd = [os.environ.get("CXX", "g++"), "-O2", "-std=c++17", "-Wall", "-I", os.path.join(HERE, "..", "include"),
           HOST_SRC, "-L", OUT_DIR, "-lpdac_b200", "-Wl,-rpath,$ORIGIN", "-o", HOST_BIN]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("host driver build failed")
    return HOST_BIN


def build(force=False, verbose=False, extra=()):
    if not force and not needs_build():
        build_host()
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    cmd = [NVCC, *FLAGS, *extra, "-o", LIB, os.path.join(CSRC, "engine.cu")]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed")
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr)
    build_host(force=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, extra=[a for a in sys.argv[1:] if a != "--force"])
