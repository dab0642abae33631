"""Builds the test-only native libraries (tests/_build/):

  libktmath_shim.so   ktmath.h with C linkage (libm accuracy tests)
  libkt_hostcheck.so  the kernels' per-ray code compiled for the host
                      (op-order checks against the oracle without a GPU;
                      the smooth tracer and its adjoint)

and makes sure the oracle port exists.  Called by conftest.py and
__graft_entry__.build().
"""
import os
import subprocess
import sys

TESTS = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(TESTS)
BUILD = os.path.join(TESTS, "_build")
CSRC = os.path.join(ROOT, "kerrtracecpp2_b200", "csrc")
SHIM = os.path.join(BUILD, "libktmath_shim.so")
HOSTCHECK = os.path.join(BUILD, "libkt_hostcheck.so")
CUDA_INC = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.exists(d) and os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        sys.stderr.write(p.stdout + p.stderr)
        raise RuntimeError("build failed: " + " ".join(cmd))


def build_all(force=False):
    os.makedirs(BUILD, exist_ok=True)
    heads = [os.path.join(CSRC, h) for h in ("ktmath.h", "ktmath_consts.h", "kt_physics.cuh",
                                             "kt_machines.cuh", "kt_frame.h", "kt_dual.cuh",
                                             "kt_smooth.cuh", "kt_smray.cuh")]
    heads.append(os.path.join(ROOT, "include", "kerrtrace.h"))
    src = os.path.join(TESTS, "ktmath_shim.c")
    if force or _newer(SHIM, [src] + heads):
        _run(["gcc", "-O2", "-ffp-contract=off", "-march=x86-64-v3", "-fPIC", "-shared", "-o", SHIM,
              src, "-lm"])
    srcs = [os.path.join(TESTS, "kt_hostcheck.cpp"), os.path.join(CSRC, "kt_frame.cpp")]
    if force or _newer(HOSTCHECK, srcs + heads):
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-march=x86-64-v3",
              "-fopenmp", "-shared", "-I", CUDA_INC, "-o", HOSTCHECK] + srcs)
    sys.path.insert(0, ROOT)
    from oracle import build as obuild  # noqa: E402

    obuild.build_port(force)


if __name__ == "__main__":
    build_all("--force" in sys.argv)
