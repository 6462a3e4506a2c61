"""Ensembles of solvers advanced together on one GPU (les_ensemble_* of les_solver.h).

The reference tunes its model constants with a Bayesian optimiser that proposes one
parameter set per LES run (bayesian_optimizer.py:568-673).  An ensemble runs many proposed
sets at once, each member with its own grid, constants, seed and output files.
``ensemble_configs`` draws the sets of the batched-ensemble workload: CS_UNBURNED uniform in
[0.08, 0.22], the flame-acceleration strength uniform in [0, 2] x its default, the nudging
coefficient uniform in [0, 1] x its default, members alternating between the 128x64x64 and
96x48x48 grids.
"""
from __future__ import annotations

import ctypes as C
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
    """n solvers on one device stepped by one multi-stream graph per step."""

    def __init__(self, cfgs: Sequence[SolverConfig], precision: int = N.FP32, autotune: bool = True, device: int = 0,
                 chem: str = N.CHEM_BIN, tran: str = N.TRAN_BIN):
        L = N.lib()
        arr = (N.LesgpuConfig * len(cfgs))(*[N.LesgpuConfig.from_config(c, precision, device) for c in cfgs])
        h = C.c_void_p()
        rc = L.les_ensemble_create(arr, len(cfgs), chem.encode(), tran.encode(), 1 if autotune else 0, C.byref(h))
        if rc != 0:
            raise N.LesgpuError(rc, "les_ensemble_create failed")
        self._h = h
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
