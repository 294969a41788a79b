"""Build recipe of the GPU library libbh_gpu.so (sm_100a).

Compiles blackhole_b200/csrc/*.cu and *.cpp with nvcc into
blackhole_b200/lib/libbh_gpu.so.  Incremental on modification times; run as
``python -m blackhole_b200.build`` or through ``__graft_entry__.build()``.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "lib", "libbh_gpu.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3", "-I", CSRC, "-I", INCLUDE]


def _deps():
    hdrs = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh"))
    hdrs.append(os.path.join(INCLUDE, "bh_gpu.h"))
    return hdrs


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    objs = []
    hdrs = _deps()
    for s in srcs:
        o = os.path.join(BUILD, os.path.basename(s) + ".o")
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            cmd = [NVCC] + ARCH + COMMON + ["-c", s, "-o", o]
            if s.endswith(".cu"):
                cmd += ["-Xptxas", "-v"]
            r = subprocess.run(cmd, capture_output=True, text=True)
            log = os.path.join(BUILD, os.path.basename(s) + ".log")
            with open(log, "w") as f:
                f.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
            if r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
                raise RuntimeError(f"nvcc failed on {s} (see {log})")
            if verbose:
                print(f"compiled {os.path.basename(s)}")
    if force or _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart_static", "-lrt", "-lpthread", "-ldl"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("nvcc link failed")
        if verbose:
            print(f"linked {LIB}")
    build_check(verbose=verbose, force=force)
    return LIB


# Test harness library: the adjoint's per-ray code compiled for the host (the
# tests check its mathematics on a CPU); never loaded by the render library.
CHECK_LIB = os.path.join(HERE, "lib", "libbh_adjoint_check.so")


def build_check(verbose: bool = False, force: bool = False) -> str:
    srcs = [os.path.join(CSRC, "check", "bh_adjoint_check.cu"), os.path.join(CSRC, "bh_scene.cpp"),
            os.path.join(CSRC, "bh_adjoint_frame.cpp")]
    hdrs = _deps()
    objs = []
    for s in srcs:
        o = os.path.join(BUILD, "check_" + os.path.basename(s) + ".o")
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            cmd = [NVCC] + ARCH + COMMON + ["-c", s, "-o", o]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
                raise RuntimeError(f"nvcc failed on {s}")
            if verbose:
                print(f"compiled {os.path.basename(s)} (check)")
    if force or _stale(CHECK_LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", CHECK_LIB] + objs + ["-lcudart_static", "-lrt", "-lpthread", "-ldl"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("nvcc link failed (check library)")
        if verbose:
            print(f"linked {CHECK_LIB}")
    return CHECK_LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
