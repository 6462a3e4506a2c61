"""The C examples of the integration notes compile against include/*.h (syntax and types;
gcc -fsyntax-only, no GPU).  The first example is written against the reference's own
globals: it is spliced into the reference source by tests/dropin/build_dropin.py and
compiled there (below, when the reference source is present; tests/test_gpu_dropin.py runs
the result on a GPU).  The others are wrapped in a function with the few names they take as
given."""
import os
import re
import shutil
import subprocess

import pytest

from conftest import ROOT

PRELUDE = """#include <stdio.h>
#include "les_gpu.h"
#include "les_solver.h"
#include "les_serve.h"
void example(const lesgpu_config* cfgs, int n_trials, char** trial_dir, int start_step, int total_steps) {
"""


def c_blocks():
    with open(os.path.join(ROOT, "INTEGRATION.md")) as f:
        txt = f.read()
    return re.findall(r"```c\n(.*?)```", txt, flags=re.S)


def test_examples_compile(tmp_path):
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("gcc not available")
    blocks = c_blocks()
    assert len(blocks) >= 4
    for n, b in enumerate(blocks[1:], 1):
        body = "\n".join(l for l in b.splitlines() if not l.startswith("#include"))
        # `cfg` of the later examples stands for the one built in the first
        body = body.replace("lesgpu_config cfg = { /* as above */ };", "lesgpu_config cfg = cfgs[0];")
        if "lesgpu_config cfg" not in body:
            body = "lesgpu_config cfg = cfgs[0]; (void)cfg;\n" + body
        src = tmp_path / f"ex{n}.c"
        src.write_text(PRELUDE + body + "\n}\n")
        r = subprocess.run([gcc, "-fsyntax-only", "-std=c11", "-Wall", "-Wno-unused-variable",
                            "-Wno-unused-but-set-variable", "-I", os.path.join(ROOT, "include"), str(src)],
                           capture_output=True, text=True)
        assert r.returncode == 0, f"example {n}:\n{r.stderr}"


def test_first_example_compiles_inside_the_reference(tmp_path):
    """The drop-in block of the first example, spliced into the reference's own source, is
    valid C against les_gpu.h (every patch site matched exactly once)."""
    import sys
    sys.path.insert(0, os.path.join(ROOT, "tests", "dropin"))
    import build_dropin
    ref = build_dropin.build_ref.default_ref()
    src_path = os.path.join(ref, "les_combustion_solver.c")
    if not os.path.exists(src_path) or shutil.which("gcc") is None:
        pytest.skip("reference source or gcc not present")
    with open(src_path, encoding="utf-8") as f:
        patched = build_dropin.patch_dropin(f.read(), build_dropin.build_ref.CONFIGS["c1"])
    assert "gpu_step(t_loop, &DT_sim, &max_velocity)" in patched
    assert "calculate_RHS(t_loop, u_temp" not in patched.split("for (int t_loop")[1].split("lesgpu_destroy")[0]
    src = tmp_path / "dropin.c"
    src.write_text(patched)
    r = subprocess.run(["gcc", "-fsyntax-only", "-fopenmp", "-w", "-I", os.path.join(ROOT, "include"), str(src)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
