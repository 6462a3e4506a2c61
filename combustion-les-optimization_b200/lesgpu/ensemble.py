"""Ensembles of solvers advanced together on one GPU (les_ensemble_* of les_solver.h).

The reference tunes its model constants with a Bayesian optimiser that proposes one
parameter set per LES run (bayesian_optimizer.py:568-673).  An ensemble runs many proposed
sets at once, each member with its own grid, constants, seed and output files.
``ensemble_configs`` draws the sets of the batched-ensemble workload: CS_UNBURNED uniform in
[0.08, 0.22], the flame-acceleration strength uniform in [0, 2] x its default, the nudging
coefficient uniform in [0, 1] x its default, members alternating between the 128x64x64 and
96x48x48 grids.

Measurement (one JSON line; wall time of a long run, set-up of each run included):

    python -m lesgpu.ensemble --members 64 --precision fp32 --steps 200 [--sequential]
"""
from __future__ import annotations

import ctypes as C
import json
import time
from collections import Counter
from typing import List, Sequence

import numpy as np

from . import native as N
from .config import PRESETS, SolverConfig

_DEFAULT = SolverConfig()


def ensemble_configs(n: int = 64, seed: int = 2024, grids: Sequence[str] = ("e128", "e96")) -> List[SolverConfig]:
    rng = np.random.default_rng(seed)
    cs = rng.uniform(0.08, 0.22, n)
    strength = rng.uniform(0.0, 2.0, n) * _DEFAULT.accel_strength
    relax = rng.uniform(0.0, 1.0, n) * _DEFAULT.relax
    return [PRESETS[grids[q % len(grids)]].replace(cs_unburned=float(cs[q]), accel_strength=float(strength[q]),
                                                   relax=float(relax[q]), seed=int(seed + 17 * q + 1))
            for q in range(n)]


class Ensemble:
    """n solvers on one device stepped by one CUDA graph per step: a multi-stream graph of
    every member's kernels, or (batched=True) one launch per RK pass for all members of one
    grid shape (lesgpu_group_create_batched)."""

    def __init__(self, cfgs: Sequence[SolverConfig], precision: int = N.FP32, autotune: bool = True, device: int = 0,
                 chem: str = N.CHEM_BIN, tran: str = N.TRAN_BIN, batched: bool = False, per_batch: int = 0):
        L = N.lib()
        arr = (N.LesgpuConfig * len(cfgs))(*[N.LesgpuConfig.from_config(c, precision, device) for c in cfgs])
        h = C.c_void_p()
        rc = L.les_ensemble_create(arr, len(cfgs), chem.encode(), tran.encode(), 1 if autotune else 0, C.byref(h))
        if rc != 0:
            raise N.LesgpuError(rc, "les_ensemble_create failed")
        self._h = h
        if batched:
            rc = L.les_ensemble_set_batched(h, 1, per_batch)
            if rc != 0:
                raise N.LesgpuError(rc, "les_ensemble_set_batched failed")
        self.cfgs = list(cfgs)
        self.members = [N.Solver.wrap(L.les_ensemble_member(h, q), c) for q, c in enumerate(self.cfgs)]

    def run(self, nsteps: int, chunk: int = 64):
        rc = N.lib().les_ensemble_run(self._h, nsteps, chunk)
        if rc != 0:
            raise N.LesgpuError(rc, N.lib().les_ensemble_last_error(self._h).decode())

    @property
    def cells(self) -> int:
        return sum(c.cells for c in self.cfgs)

    def close(self):
        if getattr(self, "_h", None):
            for m in self.members:
                m.close()
            N.lib().les_ensemble_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _timed(f) -> float:
    """Wall seconds of f(); every call into the library returns after the device finished."""
    t = time.perf_counter()
    f()
    return time.perf_counter() - t


def main(argv=None) -> int:
    import argparse
    ap = argparse.ArgumentParser(description="Time an ensemble of solvers stepped by one multi-stream graph")
    ap.add_argument("--members", type=int, default=64)
    ap.add_argument("--grids", default="e128,e96", help="comma-separated presets, assigned round-robin")
    ap.add_argument("--precision", choices=["fp64", "fp32"], default="fp32")
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--chunk", type=int, default=64)
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--batched", action="store_true",
                    help="one launch per RK pass for all members of a grid shape instead of the multi-stream graph")
    ap.add_argument("--per-batch", type=int, default=0, help="with --batched: at most this many members per launch")
    ap.add_argument("--sequential", action="store_true",
                    help="also time one solo solver per grid and sum them over the members")
    a = ap.parse_args(argv)
    prec = N.FP32 if a.precision == "fp32" else N.FP64
    grids = tuple(a.grids.split(","))
    cfgs = ensemble_configs(a.members, grids=grids)
    out = {"members": a.members, "grids": dict(Counter(grids[q % len(grids)] for q in range(a.members))),
           "precision": a.precision, "steps": a.steps, "chunk": a.chunk, "autotune": not a.no_autotune,
           "form": f"batched (max {a.per_batch or 'all'} per launch)" if a.batched else "multi-stream"}
    t = time.perf_counter()
    ens = Ensemble(cfgs, precision=prec, autotune=not a.no_autotune, batched=a.batched, per_batch=a.per_batch)
    out["create_s"] = time.perf_counter() - t
    tiles = {}
    for q, m in enumerate(ens.members):
        tiles.setdefault(grids[q % len(grids)], Counter())[tuple(m.ctx.get_tiles())] += 1
    out["tiles"] = {g: [list(k) + [n] for k, n in c.most_common()] for g, c in tiles.items()}
    if a.warmup:
        ens.run(a.warmup, chunk=a.chunk)
    w = _timed(lambda: ens.run(a.steps, chunk=a.chunk))
    out["ms_per_step"] = w * 1e3 / a.steps
    out["cells"] = ens.cells
    out["cell_steps_per_s"] = ens.cells * a.steps / w
    out["finite"] = all(bool(np.isfinite(m.state()["u"]).all()) for m in ens.members)
    ens.close()
    if a.sequential:
        solo = {}
        for g in grids:
            q = grids.index(g)
            s = N.Solver(cfgs[q], precision=prec)
            if not a.no_autotune:
                s.ctx.autotune(3)
            s.run_device(a.warmup or 1, chunk=a.chunk)
            solo[g] = _timed(lambda: s.run_device(a.steps, chunk=a.chunk)) * 1e3 / a.steps
            s.close()
        seq = sum(solo[grids[q % len(grids)]] for q in range(a.members))
        out["solo_ms_per_step"] = solo
        out["sequential_ms_per_step"] = seq
        out["speedup_vs_sequential"] = seq / out["ms_per_step"]
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
