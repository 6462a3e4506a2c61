"""Error of the FP32 precision form against the FP64 form, stated per output profile.

Runs one case twice on the GPU -- the plain FP64 form and the FP32-bulk form (fields and
stencil arithmetic in FP32; global sums, maxima, dt and the SEM inflow in FP64) -- from the
same initial state and the same rand() stream, with the probe files on, then compares the
profile statistics of ``stats`` computed from each run's probe rows (all stations pooled)
and the final state fields.

The flow is chaotic: any perturbation, even at rounding level, grows until the two
trajectories decorrelate, after which their statistics differ by sampling noise alone.  A
further FP64 runs from an initial field scaled by (1 + eps) separate that floor from the
precision error: eps = 1e-15 (rounding level in FP64) and eps = 1e-7 (rounding level in FP32,
applied once).  Their profile and state differences against the first FP64 run are reported
beside the FP32 ones (``profiles_floor_<eps>``).  The scaled field is T by default; T and Y
are nudged towards their targets, so a T perturbation reaches the velocity only through the
density, while ``--floor-field u`` perturbs the velocity itself and so measures how fast the
flow amplifies a rounding-size difference.
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


def run_form(cfg: SolverConfig, precision: int, steps: int, directory: str, chunk: int = 64, device: int = 0,
             perturb: float = 0.0, field: str = "T"):
    s = N.Solver(cfg, precision=precision, device=device)
    if perturb:
        st = s.state()
        st[field] = st[field] * (1.0 + perturb)
        s.ctx.upload_state(st)
    s.set_outputs(directory, N.LES_OUT_PROBES | N.LES_OUT_MONITOR)
    t = time.perf_counter()
    s.run_device(steps, chunk=chunk)
    s.ctx.sync()
    wall = time.perf_counter() - t
    st = s.state()
    s.close()
    return st, wall


def _state_err(a, b):
    out = {}
    for f in N.STATE_NAMES:
        nb = np.linalg.norm(b[f])
        out[f] = float(np.linalg.norm(a[f] - b[f]) / (nb if nb > 0 else 1.0))
    return out


def compare(cfg: SolverConfig, steps: int, workdir: Optional[str] = None, chunk: int = 64,
            floor=(1e-15, 1e-7), floor_field: str = "T") -> dict:
    workdir = workdir or tempfile.mkdtemp(prefix="lesprec_")
    dirs = {k: os.path.join(workdir, k) for k in ("fp64", "fp32")}
    for d in dirs.values():
        os.makedirs(d, exist_ok=True)
    s64, w64 = run_form(cfg, N.FP64, steps, dirs["fp64"], chunk)
    s32, w32 = run_form(cfg, N.FP32, steps, dirs["fp32"], chunk)
    r64, r32 = _pool(dirs["fp64"]), _pool(dirs["fp32"])
    out = {"grid": [cfg.nx, cfg.ny, cfg.nz], "steps": steps, "rows_fp64": int(len(r64["u"])),
           "rows_fp32": int(len(r32["u"])), "wall_s": {"fp64": w64, "fp32": w32},
           "profiles_fp32": stats.compare_profiles(r32, r64), "state_rel_l2_fp32": _state_err(s32, s64)}
    for eps in (floor or ()):
        d = os.path.join(workdir, f"fp64_eps{eps:g}")
        os.makedirs(d, exist_ok=True)
        salt, walt = run_form(cfg, N.FP64, steps, d, chunk, perturb=eps, field=floor_field)
        ralt = _pool(d)
        out["wall_s"][f"fp64_eps{eps:g}"] = walt
        out[f"profiles_floor_{eps:g}"] = stats.compare_profiles(ralt, r64)
        out[f"state_rel_l2_floor_{eps:g}"] = _state_err(salt, s64)
    return out


def main(argv=None) -> int:
    import argparse
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--workload", default="c1")
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--chunk", type=int, default=64)
    ap.add_argument("--workdir", default=None)
    ap.add_argument("--no-floor", action="store_true")
    ap.add_argument("--floor-field", choices=["T", "u"], default="T", help="field the floor runs scale by 1 + eps")
    a = ap.parse_args(argv)
    print(json.dumps(compare(preset(a.workload), a.steps, a.workdir, a.chunk, floor=() if a.no_floor else (1e-15, 1e-7),
                             floor_field=a.floor_field)))
    return 0


if __name__ == "__main__":
    sys.exit(main())
