"""Error of the FP32 precision form against the FP64 form, stated per output profile.

Runs one case twice on the GPU -- the plain FP64 form and the FP32-bulk form (fields and
stencil arithmetic in FP32; global sums, maxima, dt and the SEM inflow in FP64) -- from the
same initial state and the same rand() stream, with the probe files on, then compares the
profile statistics of ``stats`` computed from each run's probe rows (all stations pooled,
and per station), plus the final state fields.
"""
from __future__ import annotations

import json
import os
import sys
import tempfile
import time
from typing import Dict, Optional

import numpy as np

from . import native as N
from . import stats
from .config import SolverConfig, preset


def _pool(directory: str) -> Dict[str, np.ndarray]:
    parts = []
    for loc in range(7):
        p = os.path.join(directory, f"probe_data_flame_region_loc{loc}.csv")
        if os.path.exists(p):
            r = stats.read_probe_csv(p)
            if len(r["u"]):
                parts.append(r)
    if not parts:
        return {c: np.zeros(0) for c in stats.COLUMNS}
    return {c: np.concatenate([r[c] for r in parts]) for c in stats.COLUMNS}


def run_form(cfg: SolverConfig, precision: int, steps: int, directory: str, chunk: int = 64, device: int = 0):
    s = N.Solver(cfg, precision=precision, device=device)
    s.set_outputs(directory, N.LES_OUT_PROBES | N.LES_OUT_MONITOR)
    t = time.perf_counter()
    s.run_device(steps, chunk=chunk)
    s.ctx.sync()
    wall = time.perf_counter() - t
    st = s.state()
    s.close()
    return st, wall


def compare(cfg: SolverConfig, steps: int, workdir: Optional[str] = None, chunk: int = 64) -> dict:
    workdir = workdir or tempfile.mkdtemp(prefix="lesprec_")
    d64, d32 = os.path.join(workdir, "fp64"), os.path.join(workdir, "fp32")
    os.makedirs(d64, exist_ok=True)
    os.makedirs(d32, exist_ok=True)
    s64, w64 = run_form(cfg, N.FP64, steps, d64, chunk)
    s32, w32 = run_form(cfg, N.FP32, steps, d32, chunk)
    r64, r32 = _pool(d64), _pool(d32)
    out = {"grid": [cfg.nx, cfg.ny, cfg.nz], "steps": steps, "rows_fp64": int(len(r64["u"])),
           "rows_fp32": int(len(r32["u"])), "wall_s": {"fp64": w64, "fp32": w32},
           "profiles_pooled": stats.compare_profiles(r32, r64), "state_rel_l2": {}}
    for f in N.STATE_NAMES:
        a, b = s32[f], s64[f]
        nb = np.linalg.norm(b)
        out["state_rel_l2"][f] = float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))
    return out


def main(argv=None) -> int:
    import argparse
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--workload", default="c1")
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--chunk", type=int, default=64)
    ap.add_argument("--workdir", default=None)
    a = ap.parse_args(argv)
    print(json.dumps(compare(preset(a.workload), a.steps, a.workdir, a.chunk)))
    return 0


if __name__ == "__main__":
    sys.exit(main())
