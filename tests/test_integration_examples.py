"""The C examples of the integration notes compile against include/*.h (syntax and types;
gcc -fsyntax-only, no GPU).  The first example uses the reference's own globals and is
skipped; the others are wrapped in a function with the few names they take as given."""
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
