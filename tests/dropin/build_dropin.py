#!/usr/bin/env python3
"""Build the reference solver with its loop body replaced by the C-ABI calls (test harness).

This is the drop-in a maintainer of the reference would make, done mechanically so a test can
run it: ``les_combustion_solver.c`` from the reference checkout gets

* the oracle recipe's patch (``oracle/build_ref.py``: grid and model constants for a named
  grid, seeded ``srand``, ``OUTPUT_DIR "./"``, step count from the environment, state dumps
  after each step),
* the first C block of ``INTEGRATION.md`` -- ``gpu_begin`` / ``gpu_step`` -- inserted
  verbatim before ``main()``,
* three edits in ``main()``: ``gpu_begin(...)`` before the time loop, the loop body from the
  in-loop ``calculate_max_velocity`` (``les_combustion_solver.c:4399``) through
  ``apply_boundary_conditions`` (``:4555``) replaced by ``gpu_step(...)``, and
  ``lesgpu_destroy`` after the loop;

and is compiled with the reference's flags against ``liblesgpu.so``.  The binary goes to
``tests/dropin/_build/<grid>/les_dropin`` beside copies of ``chem.bin`` / ``tran.bin``.  The
reference tree is only read.  Usage::

    python tests/dropin/build_dropin.py [--ref /path/to/reference] [--config c1]
"""
from __future__ import annotations

import argparse
import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
PKG = os.path.join(ROOT, "combustion-les-optimization_b200")
OUT_ROOT = os.path.join(HERE, "_build")
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import build_ref  # noqa: E402


def integration_block() -> str:
    """The first ```c block of INTEGRATION.md (the code a maintainer adds to the reference)."""
    with open(os.path.join(ROOT, "INTEGRATION.md"), encoding="utf-8") as f:
        txt = f.read()
    blocks = re.findall(r"```c\n(.*?)```", txt, flags=re.S)
    if not blocks or "gpu_step" not in blocks[0]:
        raise RuntimeError("INTEGRATION.md: first C block with gpu_begin/gpu_step not found")
    return blocks[0]


def _sub1(src: str, pattern: str, repl, flags=0) -> str:
    new, n = re.subn(pattern, repl, src, flags=flags)
    if n != 1:
        raise RuntimeError(f"drop-in patch {pattern!r} matched {n} times (expected exactly 1)")
    return new


def patch_dropin(ref_src: str, cfg: dict) -> str:
    s = build_ref.patch_source(ref_src, cfg)
    block = integration_block()
    s = _sub1(s, r"^int main\(int argc, char \*argv\[\]\) \{",
              lambda m: "/* ---- drop-in (INTEGRATION.md, first C block) ---- */\n" + block
              + "\n/* ---- end of drop-in ---- */\n" + m.group(0), flags=re.M)
    begin = ("if (gpu_begin(les_ref_seed, CS_UNBURNED, CS_BURNT, CS_FLAME_BOOST, FLAME_ACCEL_STRENGTH,"
             " FLAME_ACCEL_WIDTH, FLAME_ACCEL_CENTER, les_ref_relax) != 0) { fprintf(stderr, \"gpu_begin failed\\n\");"
             " return 1; }\n    ")
    s = _sub1(s, r'printf\("\\n--- Simulation Loop Start ---\\n"\);', lambda m: begin + m.group(0))
    # the in-loop dt block (its calculate_max_velocity is followed by DT_conv) through the
    # boundary conditions, whose line the oracle patch ends with the per-step dump hook
    s = _sub1(s, r"calculate_max_velocity\(attribute, u, v, w, &max_velocity\);\s*\n\s*double DT_conv.*?"
                 r"apply_boundary_conditions\(attribute, u, v, w, rhou, rhov, rhow, G, T, P, Yk, rho\);"
                 r" les_ref_after_step\(t_loop, DT_sim\);",
              lambda m: "if (gpu_step(t_loop, &DT_sim, &max_velocity) != LESGPU_OK) break;"
                        " les_ref_after_step(t_loop, DT_sim);", flags=re.S)
    s = _sub1(s, r'printf\("\\nFinalizing output\.\.\.\\n"\);', lambda m: "lesgpu_destroy(gpu);\n    " + m.group(0))
    return s


def _cuda_lib_dir() -> str:
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    base = os.path.dirname(os.path.dirname(os.path.realpath(nvcc)))
    for d in ("lib64", "targets/x86_64-linux/lib"):
        if os.path.exists(os.path.join(base, d, "libcudart.so")):
            return os.path.join(base, d)
    return os.path.join(base, "lib64")


def build(ref_dir: str, names=("c1",), quiet: bool = False) -> None:
    lib = os.path.join(PKG, "liblesgpu.so")
    if not os.path.exists(lib):
        raise FileNotFoundError(f"{lib} missing: build the package first")
    with open(os.path.join(ref_dir, "les_combustion_solver.c"), encoding="utf-8") as f:
        ref_src = f.read()
    for name in names:
        out = os.path.join(OUT_ROOT, name)
        os.makedirs(out, exist_ok=True)
        csrc = os.path.join(out, "les_dropin.c")
        with open(csrc, "w", encoding="utf-8") as f:
            f.write(patch_dropin(ref_src, build_ref.CONFIGS[name]))
        for fn in ("chem.bin", "tran.bin"):
            shutil.copyfile(os.path.join(PKG, "data", fn), os.path.join(out, fn))
        exe = os.path.join(out, "les_dropin")
        cuda_lib = _cuda_lib_dir()
        # the library is found relative to the binary, so the tree can move (it does, to the GPU box)
        rel_pkg = os.path.relpath(PKG, out)
        cmd = ["gcc", "-O2", "-fopenmp", "-ffp-contract=off", "-w", "-I", os.path.join(ROOT, "include"), csrc,
               "-o", exe, "-L", PKG, "-llesgpu", f"-Wl,-rpath,$ORIGIN/{rel_pkg}", "-L", cuda_lib,
               f"-Wl,-rpath,{cuda_lib}", "-lcudart", "-lm"]
        subprocess.run(cmd, check=True)
        if not quiet:
            print(f"built {exe}")


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--ref", default=build_ref.default_ref())
    ap.add_argument("--config", action="append", choices=sorted(build_ref.CONFIGS))
    a = ap.parse_args(argv)
    build(a.ref, a.config or ["c1"])
    return 0


if __name__ == "__main__":
    sys.exit(main())
