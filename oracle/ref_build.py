"""Build recipe for ``oracle/_ref``: the reference's own sources, compiled here.

Test infrastructure only.  Nothing in the product path imports or links this.

The artefacts, written only into ``oracle/_ref/``, are

* ``refgpu_<variant>`` -- the same kernels compiled by nvcc for sm_100a and
  launched on the GPU as the reference's serial main launches them
  (``oracle/refgpu_harness.cu``), for GPU-against-GPU parity and a timing of
  the reference's kernels on the same device.
* ``librefk_<variant>.so`` -- the reference's CUDA kernel sources
  (``src/k_stream_collide_stream.c``, ``src/k_collide.c``,
  ``src/system_boundary_kernels.c`` and the device helpers in
  ``src/lattice.c``) compiled as plain C for the CPU through
  ``oracle/refk_harness.c``, which runs every launch as a sequential loop over
  blocks of one thread.  The AA-pattern kernels touch a disjoint slot set per
  node, so the sequential run computes what the GPU launch computes (up to FMA
  contraction on the GPU).  They pin the C restatement and, run on the
  host cores, are the reference arm of bench.py.

A build variant is a set of ``flags.h`` values.  ``flags.h`` has one include
guard and no per-flag guards, so each variant gets an edited copy written to
``oracle/_ref/<variant>/flags.h`` (never committed) and force-included ahead of
the reference sources, which makes the reference's own ``#include "flags.h"``
a no-op.  The sources themselves are compiled where they lie.

Usage:  python oracle/ref_build.py [--src DIR]   (needs the reference tree)
"""
from __future__ import annotations

import argparse
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")


def reference_root() -> str:
    """The reference project's checkout: $LBX_REFERENCE_ROOT, else a directory
    named `reference` beside this repository."""
    env = os.environ.get("LBX_REFERENCE_ROOT")
    if env:
        return env
    return os.path.normpath(os.path.join(HERE, "..", "..", "reference"))


DEFAULT_SRC = os.path.join(reference_root(), "src")

# name -> flags.h overrides.  PEST output is off except in the *_pest
# variants: with it on and no PEST input files the reference dereferences a
# never-allocated buffer.
VARIANTS = {
    "d2q9_f64": dict(NUM_DIMENSIONS=2, NUM_FLUID_COMPONENTS=1, DP_ON=1),
    "d2q9_f32": dict(NUM_DIMENSIONS=2, NUM_FLUID_COMPONENTS=1, DP_ON=0),
    "d3q19_f64": dict(NUM_DIMENSIONS=3, NUM_FLUID_COMPONENTS=1, DP_ON=1),
    "d3q19_f32": dict(NUM_DIMENSIONS=3, NUM_FLUID_COMPONENTS=1, DP_ON=0),
    "d2q9s_f64": dict(NUM_DIMENSIONS=2, NUM_FLUID_COMPONENTS=2, DP_ON=1),
    "d3q19s_f64": dict(NUM_DIMENSIONS=3, NUM_FLUID_COMPONENTS=2, DP_ON=1),
    "d3q19s_f32": dict(NUM_DIMENSIONS=3, NUM_FLUID_COMPONENTS=2, DP_ON=0),
    # plain compressible BGK ("ACCURATE 0, COMPRESSIBLE 1")
    "d3q19p_f64": dict(NUM_DIMENSIONS=3, NUM_FLUID_COMPONENTS=1, DP_ON=1,
                       ACCURATE=0, COMPRESSIBLE=1),
    "d2q9p_f64": dict(NUM_DIMENSIONS=2, NUM_FLUID_COMPONENTS=1, DP_ON=1,
                      ACCURATE=0, COMPRESSIBLE=1),
    # shifted compressible ("ACCURATE 1, COMPRESSIBLE 1")
    "d3q19c_f64": dict(NUM_DIMENSIONS=3, NUM_FLUID_COMPONENTS=1, DP_ON=1,
                       ACCURATE=1, COMPRESSIBLE=1),
    "d3q19p_f32": dict(NUM_DIMENSIONS=3, NUM_FLUID_COMPONENTS=1, DP_ON=0,
                       ACCURATE=0, COMPRESSIBLE=1),
    "d2q9p_f32": dict(NUM_DIMENSIONS=2, NUM_FLUID_COMPONENTS=1, DP_ON=0,
                      ACCURATE=0, COMPRESSIBLE=1),
    "d2q9s_f32": dict(NUM_DIMENSIONS=2, NUM_FLUID_COMPONENTS=2, DP_ON=0),
    # compensated (Kahan) density sums
    "d3q19k_f32": dict(NUM_DIMENSIONS=3, NUM_FLUID_COMPONENTS=1, DP_ON=0, KAHAN_SUMMATION=1),
    "d3q19k_f64": dict(NUM_DIMENSIONS=3, NUM_FLUID_COMPONENTS=1, DP_ON=1, KAHAN_SUMMATION=1),
    "d2q9k_f32": dict(NUM_DIMENSIONS=2, NUM_FLUID_COMPONENTS=1, DP_ON=0, KAHAN_SUMMATION=1),
    "d3q19sk_f32": dict(NUM_DIMENSIONS=3, NUM_FLUID_COMPONENTS=2, DP_ON=0, KAHAN_SUMMATION=1),
    # Walsh partial bounce-back (needs computing on solid nodes)
    "d3q19w_f64": dict(NUM_DIMENSIONS=3, NUM_FLUID_COMPONENTS=1, DP_ON=1,
                       COMPUTE_ON_SOLIDS=1, WALSH_NS_ON=1),
    "d3q19w_f32": dict(NUM_DIMENSIONS=3, NUM_FLUID_COMPONENTS=1, DP_ON=0,
                       COMPUTE_ON_SOLIDS=1, WALSH_NS_ON=1),
    "d2q9w_f64": dict(NUM_DIMENSIONS=2, NUM_FLUID_COMPONENTS=1, DP_ON=1,
                      COMPUTE_ON_SOLIDS=1, WALSH_NS_ON=1),
    "d3q19sw_f64": dict(NUM_DIMENSIONS=3, NUM_FLUID_COMPONENTS=2, DP_ON=1,
                        COMPUTE_ON_SOLIDS=1, WALSH_NS_ON=1),
    # PEST point sampling on (the tests supply its input files)
    "d2q9s_pest_f64": dict(NUM_DIMENSIONS=2, NUM_FLUID_COMPONENTS=2, DP_ON=1,
                           PEST_OUTPUT_ON=1),
    "d3q19s_pest_f32": dict(NUM_DIMENSIONS=3, NUM_FLUID_COMPONENTS=2, DP_ON=0,
                            PEST_OUTPUT_ON=1),
}

def variant_flags(src: str, overrides: dict) -> str:
    with open(os.path.join(src, "flags.h")) as fh:
        text = fh.read()
    overrides = dict(overrides)
    overrides.setdefault("PEST_OUTPUT_ON", 0)
    overrides.setdefault("VERBOSITY_LEVEL", 0)
    overrides.setdefault("SAY_HI", 0)
    for name, value in overrides.items():
        pat = re.compile(r"^#define\s+%s\s+.*$" % name, re.M)
        if not pat.search(text):
            raise SystemExit("flag %s not found in flags.h" % name)
        text = pat.sub("#define %s %s" % (name, value), text, count=1)
    return text


def sh(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def build(src: str, only=None) -> None:
    os.makedirs(OUT, exist_ok=True)
    for name, ov in VARIANTS.items():
        if only and name not in only:
            continue
        vdir = os.path.join(OUT, name)
        os.makedirs(vdir, exist_ok=True)
        fl = os.path.join(vdir, "flags.h")
        with open(fl, "w") as fh:
            fh.write(variant_flags(src, ov))
        sh(["gcc", "-O2", "-fPIC", "-shared", "-std=gnu99", "-w",
            "-ffp-contract=off", "-fvisibility=hidden",
            "-ffunction-sections", "-fdata-sections",
            "-Wl,--gc-sections", "-Wl,-z,defs",
            "-include", fl, "-I", src,
            os.path.join(HERE, "refk_harness.c"),
            "-o", os.path.join(OUT, "librefk_%s.so" % name), "-lm"])


# The reference's CUDA step kernels, compiled for sm_100a by nvcc into
# oracle/_ref/refgpu_<variant> through oracle/refgpu_harness.cu.
GPU_VARIANTS = ["d3q19_f32", "d3q19_f64", "d2q9_f64"]


def build_gpu(src: str, only=None) -> None:
    os.makedirs(OUT, exist_ok=True)
    for name in GPU_VARIANTS:
        if only and name not in only:
            continue
        vdir = os.path.join(OUT, name)
        os.makedirs(vdir, exist_ok=True)
        fl = os.path.join(vdir, "flags.h")
        with open(fl, "w") as fh:
            fh.write(variant_flags(src, VARIANTS[name]))
        sh(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-w",
            "-include", fl, "-I", src, os.path.join(HERE, "refgpu_harness.cu"),
            "-o", os.path.join(OUT, "refgpu_%s" % name)])


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--src", default=DEFAULT_SRC)
    ap.add_argument("--only", nargs="*")
    a = ap.parse_args(argv)
    if not os.path.isdir(a.src):
        print("reference tree not present; oracle/_ref not rebuilt")
        return 0
    build(a.src, a.only)
    build_gpu(a.src, a.only)
    return 0


if __name__ == "__main__":
    sys.exit(main())
