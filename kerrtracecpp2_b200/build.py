"""Build the renderer in-tree: kerrtracecpp2_b200/libkerrtrace.so (CUDA
kernels for sm_100a + the C ABI) and kerrtracecpp2_b200/bin/kerr_tracer (the
CLI).  nvcc cross-compiles without a GPU.

Floating-point flags matter here: the parity bar with the reference's CPU
path is bit equality, so device code is compiled with --fmad=false and host
code with -ffp-contract=off (no multiply-add contraction anywhere the
reference has a separate multiply and add).

Usage: python kerrtracecpp2_b200/build.py [--force] [--verbose]
"""
import argparse
import concurrent.futures
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libkerrtrace.so")
CLI = os.path.join(PKG, "bin", "kerr_tracer")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-std=c++17", "--fmad=false", "-lineinfo", "-Xptxas", "-v",
                     "-Xcompiler", "-fPIC,-ffp-contract=off"]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-Wall", "-Wextra",
             "-I", os.path.join(CUDA_HOME, "include")]

CU_SOURCES = ["kt_kernels.cu", "kt_noalloc.cu", "kt_mixed.cu", "kt_adjoint.cu"]
CXX_SOURCES = ["kt_frame.cpp", "kt_api.cpp", "kt_batch.cpp", "kt_grad.cpp", "kt_io.cpp",
               "kt_compat.cpp"]
HEADERS = ["ktmath.h", "ktmath_consts.h", "kt_physics.cuh", "kt_machines.cuh", "kt_internal.h",
           "kt_frame.h", "kt_context.h", "kt_trace_kernel.cuh", "kt_dual.cuh", "kt_smooth.cuh",
           "kt_smray.cuh", "kt_adjoint.h", "kt_elliptic.cuh"]
# Per-file compile flags: the exact kernels keep every multiply and add of
# the reference's arithmetic separate; the mixed-precision kernels are not
# compared bit for bit and use FMA contraction.
CU_FLAGS = {"kt_mixed.cu": ["--fmad=true"]}
# The frame set-up evaluates the independent samples of the horizon scan and
# the ISCO search on several host threads.
CXX_FILE_FLAGS = {"kt_frame.cpp": ["-fopenmp"]}


def run(cmd, verbose):
    if verbose:
        print("+", " ".join(cmd), flush=True)
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        sys.stderr.write(p.stdout + p.stderr)
        raise RuntimeError(f"command failed: {' '.join(cmd)}")
    return p.stdout + p.stderr


def newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(CLI), exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [
        os.path.join(ROOT, "include", "kerrtrace.h"),
        os.path.join(ROOT, "include", "kerrtrace_cuda_render.h")]
    objs = []
    jobs = []  # (command, is_nvcc)
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if force or newer(o, [s] + hdrs):
            flags = [f for f in NVCC_FLAGS if not (src in CU_FLAGS and f == "--fmad=false")]
            jobs.append(([NVCC] + flags + CU_FLAGS.get(src, []) + ["-c", s, "-o", o], True))
        objs.append(o)
    for src in CXX_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if force or newer(o, [s] + hdrs):
            jobs.append((["g++"] + CXX_FLAGS + CXX_FILE_FLAGS.get(src, []) + ["-c", s, "-o", o], False))
        objs.append(o)
    # Translation units compile independently: run them in parallel.
    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        outs = list(ex.map(lambda j: run(j[0], verbose), jobs))
    ptxas_log = [o for o, (_, is_nvcc) in zip(outs, jobs) if is_nvcc]
    if force or newer(LIB, objs):
        run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lgomp"], verbose)
    cli_src = os.path.join(PKG, "cli", "kerr_tracer.cpp")
    if os.path.exists(cli_src) and (force or newer(CLI, [cli_src, LIB] + hdrs)):
        run(["g++", "-O2", "-std=c++17", "-Wall", "-o", CLI, cli_src, "-L", PKG, "-lkerrtrace",
             "-Wl,-rpath,$ORIGIN/.."], verbose)
    if ptxas_log:
        with open(os.path.join(BUILD, "ptxas.log"), "w") as f:
            f.write("\n".join(ptxas_log))
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose))


if __name__ == "__main__":
    main()
