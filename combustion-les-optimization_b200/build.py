#!/usr/bin/env python3
"""Build ``liblesgpu.so`` in-tree: CUDA kernels for sm_100a plus the C host driver.

* ``csrc/les_f64.cu``  -- plain FP64 form, compiled with ``-fmad=false`` (no FMA
  contraction, matching the reference's x86-64 arithmetic operation for operation);
* ``csrc/les_f64_aux.cu`` -- SEM plane, device-loop dt / rand() draws, division self-check
  (``-fmad=false``: bit-identical to the host);
* ``csrc/les_f32.cu``  -- FP32-bulk precision form, FMA contraction on;
* ``csrc/les_api.cu``  -- the C ABI of ``include/les_gpu.h``;
* ``host/*.c``         -- the C host side (solver loop, glibc-compatible rand(), SEM vortex
  bookkeeping, probe/monitor/checkpoint files), built with ``-ffp-contract=off``.

Usage: ``python build.py [--force] [--verbose]``.  Objects go to ``_build/``.
"""
from __future__ import annotations

import argparse
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
INC = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "liblesgpu.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# Units compiled without FMA contraction: the FP64 stage kernels (the reference's operation
# order, one rounding per operation) and the shared SEM / device-loop code, whose results
# must equal the host's bit for bit.
FMAD_OFF = {"les_f64", "les_f64_aux", "les_pstat"}


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _cuda_lib_dir(nvcc: str) -> str:
    base = os.path.dirname(os.path.dirname(os.path.realpath(nvcc)))
    for d in ("lib64", "targets/x86_64-linux/lib"):
        p = os.path.join(base, d)
        if os.path.exists(os.path.join(p, "libcudart.so")) or os.path.exists(os.path.join(p, "libcudart_static.a")):
            return p
    return os.path.join(base, "lib64")


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr)
    return r


def sources():
    cu = sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))
    c = sorted(glob.glob(os.path.join(HERE, "host", "*.c")))
    hdr = (sorted(glob.glob(os.path.join(HERE, "csrc", "*.cuh"))) + sorted(glob.glob(os.path.join(HERE, "csrc", "*.h")))
           + sorted(glob.glob(os.path.join(HERE, "host", "*.h"))) + sorted(glob.glob(os.path.join(INC, "*.h"))))
    return cu, c, hdr


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    cu, c, hdr = sources()
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(p) <= t for p in cu + c + hdr + [__file__])


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False, defines=(), out: str = None,
          build_dir: str = None) -> str:
    """Compile the library.  ``defines`` (e.g. ``["LES_MINB_SCALAR=3"]``) and ``out`` build
    a variant elsewhere; the default build goes to liblesgpu.so in-tree."""
    lib_path = out or LIB
    bdir = build_dir or BUILD
    if not force and out is None and not defines and up_to_date():
        return LIB
    nvcc = _nvcc()
    os.makedirs(bdir, exist_ok=True)
    cu, c, _ = sources()
    objs = []
    for src in cu:
        name = os.path.splitext(os.path.basename(src))[0]
        obj = os.path.join(bdir, name + ".o")
        flags = [nvcc, "-c", src, "-o", obj, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                 "-I", INC, "-I", os.path.join(HERE, "csrc")] + ARCH + [f"-D{d}" for d in defines]
        flags += ["-fmad=false"] if name in FMAD_OFF else ["-fmad=true"]
        if ptxas_verbose:
            flags += ["-Xptxas", "-v"]
        r = _run(flags, verbose)
        if ptxas_verbose:
            print(r.stderr)
        objs.append(obj)
    for src in c:
        name = os.path.splitext(os.path.basename(src))[0]
        obj = os.path.join(bdir, name + ".o")
        _run(["gcc", "-c", src, "-o", obj, "-O2", "-ffp-contract=off", "-fPIC", "-std=c11", "-Wall", "-pthread",
              "-I", INC, "-I", os.path.join(HERE, "host")], verbose)
        objs.append(obj)
    tmp = lib_path + ".tmp"
    _run([nvcc, "-shared", "-o", tmp] + objs + ARCH + ["-Xcompiler", "-fPIC", "-lcudart", "-lm", "-lpthread",
                                                          "-L", _cuda_lib_dir(nvcc)], verbose)
    os.replace(tmp, lib_path)
    return lib_path


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print register/spill usage")
    a = ap.parse_args(argv)
    print(build(force=a.force, verbose=a.verbose, ptxas_verbose=a.ptxas))
    return 0


if __name__ == "__main__":
    sys.exit(main())
