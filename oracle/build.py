"""Build recipe for the oracle -- TEST INFRASTRUCTURE, not the product.

Produces:
  oracle/_build/liboracle_port.so   the C restatement (kt_oracle.c), always;
  oracle/_ref/libktref_strict.so    the reference renderer compiled from its
  oracle/_ref/libktref_stock.so     own sources (only where the reference tree
  oracle/_ref/libktref_ieee.so      exists, i.e. in the build container):
    strict: -O2 -ffp-contract=off, the renderer's libm interposed (parity),
            complex products and quotients by the textbook formulas
            (-fcx-limited-range, as the reference's own -ffast-math build
            evaluates them; only the elliptic-closed solver uses them);
    stock : the reference's own -O3 -ffast-math, glibc libm (as shipped);
    ieee  : -O3 without -ffast-math, glibc libm.  The timed CPU baseline:
            under -ffast-math (-ffinite-math-only) the reference's DOPRI5
            sentinel test std::isnan(k1_fsal.v[0]) (geodesic.hpp:321) folds
            to false, so the stock build's DOPRI5 rejects every step and
            returns each ray at the camera; the ieee build traces correctly.

The reference is compiled from a copy of its tree taken into oracle/_ref/src
(git-ignored build output, never committed) with exactly one token changed:
geodesic.hpp:326 passes the address of a C99 compound literal,
`(const double[]){a21}`, which g++ 13 rejects ("taking address of temporary
array"); it becomes `&a21`, the same value.  Nothing else is edited.

Also, with the reference tree and the renderer's library present:
  oracle/_ref/kerr_tracer_ref_cuda  the reference's own main.cpp built with
            -DUSE_CUDA, its CUDA entry point cuda_render (gpu/cuda/tracer.cuh,
            reached through a forwarding header generated in
            oracle/_ref/cuda_inc) linked from kerrtracecpp2_b200/libkerrtrace.so
            instead of gpu/cuda/tracer.cu: the drop-in link check of the
            replacement library.

The reference tree is found at --reference DIR, else at $KT_REFERENCE_DIR,
else in a directory named `reference` beside this repository.

Usage: python oracle/build.py [--reference DIR] [--force]
"""
import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
BUILD = os.path.join(HERE, "_build")
REF_OUT = os.path.join(HERE, "_ref")
DEFAULT_REFERENCE = os.environ.get("KT_REFERENCE_DIR") or os.path.join(os.path.dirname(ROOT),
                                                                        "reference")

# Files of the reference tree that main.cpp needs (its own includes).
REF_FILES = ["main.cpp", "camera.hpp", "geodesic.hpp", "knds_metric.hpp", "ray_bundle.hpp",
             "wormhole_metric.hpp", "stb_image.h", "stb_image_write.h"]
PATCH_FILE = "geodesic.hpp"
PATCH_OLD = "(const double[]){a21}"
PATCH_NEW = "&a21"

# Host ISA for every oracle build: AVX2+FMA, so the libraries built here run
# on any recent x86-64 host (the reference's own -march=native would not).
MARCH = "-march=x86-64-v3"


def run(cmd, cwd=None):
    print("+", " ".join(cmd), flush=True)
    subprocess.run(cmd, cwd=cwd, check=True)


def newer(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build_port(force=False):
    os.makedirs(BUILD, exist_ok=True)
    src = os.path.join(HERE, "kt_oracle.c")
    deps = [src, os.path.join(HERE, "kt_oracle.h"),
            os.path.join(ROOT, "kerrtracecpp2_b200", "csrc", "ktmath.h"),
            os.path.join(ROOT, "include", "kerrtrace.h")]
    out = os.path.join(BUILD, "liboracle_port.so")
    if force or newer(out, deps):
        run(["gcc", "-std=c11", "-O2", "-ffp-contract=off", MARCH, "-fopenmp", "-fPIC",
             "-shared", "-o", out, src, "-lm"])
    return out


def copy_reference(reference):
    src_dir = os.path.join(REF_OUT, "src")
    os.makedirs(src_dir, exist_ok=True)
    for f in REF_FILES:
        shutil.copyfile(os.path.join(reference, f), os.path.join(src_dir, f))
    p = os.path.join(src_dir, PATCH_FILE)
    text = open(p).read()
    if text.count(PATCH_OLD) != 1:
        raise RuntimeError(f"expected exactly one '{PATCH_OLD}' in {PATCH_FILE}")
    open(p, "w").write(text.replace(PATCH_OLD, PATCH_NEW))
    return src_dir


def build_reference(reference, force=False):
    if not os.path.isdir(reference):
        print(f"reference tree {reference} absent: using prebuilt oracle/_ref if present")
        return None
    src_dir = copy_reference(reference)
    harness = os.path.join(HERE, "ref_harness.cpp")
    interpose = os.path.join(HERE, "ref_libm_interpose.c")
    ktmath = os.path.join(ROOT, "kerrtracecpp2_b200", "csrc", "ktmath.h")
    deps = [harness, interpose, ktmath, os.path.join(ROOT, "include", "kerrtrace.h")] + \
        [os.path.join(reference, f) for f in REF_FILES]
    common = ["-std=c++17", "-fPIC", "-fopenmp", "-DOUT_DIR=\"/tmp\"", "-w", "-I", src_dir]
    strict = os.path.join(REF_OUT, "libktref_strict.so")
    if force or newer(strict, deps):
        obj = os.path.join(REF_OUT, "interpose.o")
        run(["gcc", "-std=c11", "-O2", "-ffp-contract=off", MARCH, "-fPIC", "-c",
             "-o", obj, interpose])
        run(["g++"] + common + ["-O2", "-ffp-contract=off", "-fno-builtin", "-fcx-limited-range",
                                MARCH, "-shared", "-o", strict, harness, obj, "-lm"])
    stock = os.path.join(REF_OUT, "libktref_stock.so")
    if force or newer(stock, deps):
        run(["g++"] + common + ["-O3", "-ffast-math", MARCH, "-shared", "-o", stock, harness,
                                "-lm"])
    ieee = os.path.join(REF_OUT, "libktref_ieee.so")
    if force or newer(ieee, deps):
        run(["g++"] + common + ["-O3", MARCH, "-shared", "-o", ieee, harness, "-lm"])
    build_reference_main_cuda(reference, force)
    return strict, stock, ieee


REF_CUDA_MAIN = os.path.join(REF_OUT, "kerr_tracer_ref_cuda")


def build_reference_main_cuda(reference, force=False):
    """The reference's main.cpp with -DUSE_CUDA, linked against the
    replacement library: its render dispatch (main.cpp:2413-2443) calls
    cuda_render, which the library exports with the reference's signature
    (include/kerrtrace_cuda_render.h).  Its #include "gpu/cuda/tracer.cuh"
    resolves to a generated header that includes that restatement.  PNG
    output goes to the working directory (OUT_DIR ".")."""
    lib_dir = os.path.join(ROOT, "kerrtracecpp2_b200")
    lib = os.path.join(lib_dir, "libkerrtrace.so")
    if not os.path.isdir(reference) or not os.path.exists(lib):
        return None
    src_dir = copy_reference(reference)
    inc = os.path.join(REF_OUT, "cuda_inc", "gpu", "cuda")
    os.makedirs(inc, exist_ok=True)
    hdr = os.path.join(inc, "tracer.cuh")
    text = ('// generated by oracle/build.py: the reference\'s CUDA interface, served by\n'
            '// the replacement library\n#pragma once\n#include "%s"\n'
            % os.path.join(ROOT, "include", "kerrtrace_cuda_render.h"))
    if not os.path.exists(hdr) or open(hdr).read() != text:
        open(hdr, "w").write(text)
    deps = [os.path.join(reference, f) for f in REF_FILES] + [hdr, lib,
                                                             os.path.join(ROOT, "include",
                                                                          "kerrtrace_cuda_render.h")]
    if force or newer(REF_CUDA_MAIN, deps):
        run(["g++", "-std=c++17", "-O2", "-w", "-DUSE_CUDA", "-DOUT_DIR=\".\"",
             "-I", os.path.join(REF_OUT, "cuda_inc"), "-I", src_dir, "-o", REF_CUDA_MAIN,
             os.path.join(src_dir, "main.cpp"), "-L", lib_dir, "-lkerrtrace",
             "-Wl,-rpath," + os.path.relpath(lib_dir, REF_OUT).join(["$ORIGIN/", ""]), "-lm"])
    return REF_CUDA_MAIN


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=DEFAULT_REFERENCE)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--no-port", action="store_true")
    args = ap.parse_args()
    if not args.no_port:
        build_port(args.force)
    build_reference(args.reference, args.force)


if __name__ == "__main__":
    sys.exit(main())
