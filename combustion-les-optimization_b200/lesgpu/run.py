"""Run a named case for a few steps and report per-kernel-class device times.

    python -m lesgpu.run --workload c2 --precision fp64 --steps 4 [--tiles auto|default|f,s,fl,sc,e]
                         [--loop host|device] [--kernel-times] [--outputs DIR]

The case starts from the reference's initial state (les_solver_create).  With
--kernel-times the steps run host-driven with CUDA events around every kernel class and the
per-step milliseconds are printed as one JSON line; this is also the command the committed
ncu summaries profile.
"""
from __future__ import annotations

import argparse
import json
import sys
import time

from . import native as N
from .config import preset


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--workload", default="c1")
    ap.add_argument("--precision", choices=["fp64", "fp32"], default="fp64")
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=2)
    ap.add_argument("--tiles", default="default",
                    help="auto, default, or five tile-shape indices (filter,strain,flow,scalar,eos), e.g. 0,1,2,5,0")
    ap.add_argument("--loop", choices=["host", "device"], default="host")
    ap.add_argument("--kernel-times", action="store_true")
    ap.add_argument("--staged", action="store_true", help="scalar pass through the TMA-staged kernel")
    ap.add_argument("--outputs", default=None)
    a = ap.parse_args(argv)
    prec = N.FP32 if a.precision == "fp32" else N.FP64
    cfg = preset(a.workload)
    s = N.Solver(cfg, precision=prec)
    out = {"workload": a.workload, "grid": [cfg.nx, cfg.ny, cfg.nz], "precision": a.precision}
    if a.tiles == "auto":
        tiles, ms = s.ctx.autotune(3)
        out["tiles"] = tiles
        # ms per launch, rows filter/strain/flow/scalar, one column per tile (None: not served)
        out["autotune_ms"] = [[round(float(x), 5) if x < 1e29 else None for x in row] for row in ms]
    elif a.tiles != "default":
        s.ctx.set_tiles([int(t) for t in a.tiles.split(",")])
        out["tiles"] = s.ctx.get_tiles()
    if a.staged:
        s.ctx.set_scalar_staging(True)
        out["staged"] = True
    if a.outputs:
        s.set_outputs(a.outputs, N.LES_OUT_PROBES | N.LES_OUT_MONITOR)
    run = (lambda n: s.run_device(n, chunk=max(n, 1))) if a.loop == "device" else s.step
    if a.warmup:
        run(a.warmup)
    s.ctx.sync()
    if a.kernel_times:
        s.ctx.kernel_timing(True)
    t = time.perf_counter()
    run(a.steps)
    s.ctx.sync()
    out["wall_ms_per_step"] = (time.perf_counter() - t) * 1e3 / max(a.steps, 1)
    if a.kernel_times:
        kt = s.ctx.kernel_times()
        s.ctx.kernel_timing(False)
        out["kernel_ms_per_step"] = {k: v[0] / max(a.steps, 1) for k, v in kt.items()}
        out["device_ms_per_step"] = sum(out["kernel_ms_per_step"].values())
    out["t_loop"] = s.t_loop
    s.close()
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
