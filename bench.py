#!/usr/bin/env python3
"""Benchmark of the B200 solver step: cell-steps/s on the 256x128x128 plain-FP64 case.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload c2] [--precision fp64|fp32]

A "step" is one iteration of the solver's time loop (les_combustion_solver.c:4390-4603):
dt from the device maxima, SEM vortex update and inflow noise from the host rand() stream,
the SEM plane, four RK4 stages and the boundary conditions.  Inputs are seeded synthetic
data (the reference's own initial condition with a fixed srand seed and placeholder
species properties).

* value       -- cell-steps/s of K steps with the state resident in HBM, timed with CUDA
                 events on the solver's stream (max over ranks).
* e2e         -- the same through the public solver API with host buffers: the state is
                 uploaded from pinned host memory, every step reads back its dt inputs and
                 the seven probe lines, and the final state is downloaded, all timed.
* roofline    -- the dominant kernel class: algorithmic bytes per launch / average launch
                 time (CUDA events on the solver's stream) against the measured HBM peak.
* cpu_baseline-- the reference solver itself (oracle/_ref, built from its source) on this
                 host's cores, for a bounded number of steps of the same workload.

Multi-GPU: one process per GPU under torchrun; each rank advances an independent replica
of the workload (the solve does not shard), value = all cells x steps / max rank time.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import signal
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "combustion-les-optimization_b200")
sys.path.insert(0, PKG)

METRIC = "cell-steps/s: FP64 plain vs FP32/batched at ≤1e-3 profile err; p50/p99 latency"
UNIT = "cell-steps/s"
WORKLOADS = {
    "c2": "plain FP64 drop-in, 256x128x128 grid over 0.128x0.064x0.064 m, 800 SEM eddies (10%), "
          "flame plane at x=0.03 m, CFL 0.3",
    "c1": "64x32x32 grid over 0.128x0.064x0.064 m, 200 SEM eddies (10%), flame plane at x=0.03 m, CFL 0.3",
    "c3": "512x256x256 grid, 3000 SEM eddies (15%), flame plane at x=0.03 m, CFL 0.3",
}
# Algorithmic bytes per cell for one launch of each kernel class: each field the kernel must
# read or write touched once (halos and intermediates in L2 free), averaged over the four RK
# stages.  The state Phi_n is 8-byte in both forms; the other fields take the form's size e.
def kernel_bytes_per_cell(cls: str, e: int) -> float:
    state_in = (8 + 3 * e) / 4          # stage 1 filters Phi_n, stages 2-4 the stage state
    stage_out = (3 * e + 8) / 4         # stages 1-3 write the stage state, stage 4 Phi_n+1
    return {
        "filter_props": 11 * state_in + (11 + 8) * e,        # filtered fields + 8 properties
        "strain": (7 + 4) * e,                               # u v w G rho mu nu in; nu_t S ST mu_eff out
        "rhs_flow": (8 + 4) * e,                             # 8 fields in, 4 right-hand sides out
        "rhs_scalar": (10 + 7 + 4 + 10 + 10) * e + 11 * 8 + 11 * stage_out,   # F, props, k, acc in/out, Phi_n, out
        "bc": (9 + 6) * 8,                                   # EOS pass over the FP64 state
        "sem": 0,
    }[cls]


# The CPU reference is timed on the same bounded sample in both places it is reported (the
# cpu_baseline leg of this arm and the --impl reference arm): the first REF_SAMPLE_STEPS
# steps of the workload, the first of them untimed (page faults), wall time per step.
REF_SAMPLE_STEPS = 21
REF_SAMPLE_BUDGET_S = 150.0

# Whole step, FP64: per RK stage read the stage state (11 fields), Phi_n (10) and the RK
# accumulator (10), write the accumulator (10) and the next stage state (11): 52 field
# accesses x 4 stages x 8 B = 1664 B per cell-step (832 B with 4-byte fields).
STEP_BYTES_PER_CELL = 1664
# One launch of a stage kernel processes every cell for one RK stage; its algorithmic bytes are
# that stage's share of the whole-step convention, 1664 / 4 = 416 B per cell (208 in FP32).
# The kernels' own per-launch field counts (kernel_bytes_per_cell, which add the filtered
# fields, properties and right-hand sides handed between the passes) are reported beside it.
STAGE_KERNELS = ("filter_props", "strain", "rhs_flow", "rhs_scalar")


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _traffic_table():
    """DRAM bytes per cell per launch from the committed ncu summaries (profiles/*.md lines
    of the form `traffic <kernel> <workload> <precision> <bytes_per_cell>`)."""
    out = {}
    pd = os.path.join(ROOT, "profiles")
    if not os.path.isdir(pd):
        return out
    for fn in sorted(os.listdir(pd)):
        if not fn.endswith((".md", ".txt")):
            continue
        with open(os.path.join(pd, fn)) as f:
            for line in f:
                parts = line.strip().strip("`").split()
                if len(parts) == 5 and parts[0] == "traffic":
                    try:
                        out[(parts[1], parts[2], parts[3])] = float(parts[4])
                    except ValueError:
                        pass
    return out


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        fd, self.path = tempfile.mkstemp(prefix="clocks_", suffix=".csv")
        os.close(fd)
        self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits", "-lms", "100"],
                                     stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        # wait for the first sample so that the timed region is covered from its start
        t0 = time.time()
        while time.time() - t0 < 3.0 and os.path.getsize(self.path) == 0:
            time.sleep(0.05)

    def stop(self):
        if self.proc is None:
            return None
        self.proc.send_signal(signal.SIGTERM)
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                p = [x.strip() for x in line.split(",")]
                if len(p) < 9:
                    continue
                try:
                    sm.append(float(p[1]))
                    smax = max(smax, float(p[2]))
                except ValueError:
                    continue
                for n, v in zip(names, p[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
        os.remove(self.path)
        if not sm:
            return None
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def _dist(backend: str = "nccl"):
    """Rank, local rank and world size from the torchrun environment; joins the process group
    (NCCL on the GPU box, gloo for the CPU tests) when there is more than one rank."""
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world > 1 and not dist.is_initialized():
        import datetime
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, local, world


def _max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(cells: int, steps: int, ms_local: float, world: int):
    """Replicas only: every rank advances its own copy of the workload, so the job processed
    world x cells x steps cell-steps in the slowest rank's device time."""
    ms_max = _max_over_ranks(ms_local, world)
    return ms_max, world * cells * steps / (ms_max / 1e3)


def _barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_reference_rate(workload: str, max_steps: int, budget_s: float, threads: int):
    """Time the reference solver (oracle/_ref/<workload>/les_ref) on the host cores.
    Returns (cell-steps/s, steps timed, cores, kind, sample description) or None."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from lesgpu.config import preset
    cfg = preset(workload)
    exe = os.path.join(ROOT, "oracle", "_ref", workload, "les_ref")
    if os.path.exists(exe):
        work = tempfile.mkdtemp(prefix="lesref_bench_")
        for fn in ("chem.bin", "tran.bin"):
            shutil.copyfile(os.path.join(ROOT, "oracle", "_ref", workload, fn), os.path.join(work, fn))
        env = dict(os.environ, OMP_NUM_THREADS=str(threads), LES_REF_STEPS=str(max_steps), LES_REF_SEED=str(cfg.seed),
                   LES_REF_NOVTK="1", LES_REF_DUMP_EVERY="0")
        p = subprocess.Popen([exe], cwd=work, env=env, stdout=subprocess.DEVNULL, stderr=subprocess.PIPE, text=True)
        steps = []
        t0 = time.time()
        try:
            for line in p.stderr:
                if line.startswith("LESREF_STEP"):
                    steps.append(float(line.split()[3]))
                    if len(steps) >= max_steps or time.time() - t0 > budget_s:
                        break
        finally:
            p.kill()
            p.wait()
            shutil.rmtree(work, ignore_errors=True)
        if not steps:
            return None
        timed = steps[1:] if len(steps) > 1 else steps      # the first step pays page faults
        per = sum(timed) / len(timed)
        return (cfg.cells / per, len(timed), threads, "reference",
                f"{len(timed)} of {len(steps)} steps of the {cfg.nx}x{cfg.ny}x{cfg.nz} case, "
                f"OMP_NUM_THREADS={threads}, wall time per step from omp_get_wtime")
    # restated oracle fallback (1 thread) on the same workload
    import oracle
    orc = oracle.Oracle(cfg.as_dict())
    orc.step(1)
    t0 = time.time()
    n = 0
    while n < max_steps and time.time() - t0 < budget_s:
        orc.step(1)
        n += 1
    per = (time.time() - t0) / max(n, 1)
    orc.close()
    return (cfg.cells / per, n, 1, "port", f"{n} steps of the {cfg.nx}x{cfg.ny}x{cfg.nz} case, serial oracle")


def run_reference_arm(args):
    rank, _local, world = int(os.environ.get("RANK", "0")), 0, int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    r = cpu_reference_rate(args.workload, REF_SAMPLE_STEPS, budget_s=REF_SAMPLE_BUDGET_S, threads=threads)
    if r is None:
        print(json.dumps({"impl": "reference", "unavailable": "compiled reference produced no timed steps"}))
        return 0
    rate, n, cores, kind, sample = r
    from lesgpu.config import preset
    cfg = preset(args.workload)
    line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": world,
            "steps": n, "warmup": 1, "ms_per_step": cfg.cells / rate * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOADS.get(args.workload, args.workload), "grid": [cfg.nx, cfg.ny, cfg.nz],
                       "cells": cfg.cells, "precision": "fp64", "parallelism": f"OpenMP x{cores} host threads",
                       "l2": "host caches (the reference's 174 FP64 grids stay in host memory)",
                       "tiles": None},
            "cpu_baseline": {"value": rate, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_ours(args):
    import numpy as np
    import torch
    rank, local, world = _dist()
    torch.cuda.set_device(local)
    from lesgpu import native as N
    from lesgpu.config import preset
    cfg = preset(args.workload)
    prec = N.FP32 if args.precision == "fp32" else N.FP64
    esz = 4 if prec == N.FP32 else 8
    sol = N.Solver(cfg, precision=prec, device=local)
    ctx = sol.ctx
    # thread-block tile per kernel class: timed on this GPU at the initial state
    if args.tiles == "auto":
        ctx.autotune(3)
    tiles = {k: "x".join(map(str, ctx.TILES[t])) for k, t in
             zip(["filter_props", "strain", "rhs_flow", "rhs_scalar", "eos"], ctx.get_tiles())}
    # per step: loop_pre, 2 SEM, 4 x 4 stage kernels, 4 BC, loop_post, loop_monitor, loop_tick
    per_step_launches = 1 + 2 + 16 + 4 + 3

    # ---- warm-up (device-resident loop session; graph capture happens here)
    sol.loop_begin(chunk=max(args.warmup, args.steps))
    sol.loop_run(args.warmup)
    ctx.sync()
    torch.cuda.synchronize()

    # ---- value: K device-resident steps (dt, rand() draws, SEM and the RK4 step on the GPU,
    # one CUDA graph replay per step), state resident in HBM
    clocks = Clocks(local) if rank == 0 else None
    _barrier(world)
    torch.cuda.synchronize()
    ctx.sync()
    if clocks:
        clocks.start()
    ctx.mark(0)
    sol.loop_run(args.steps)
    ctx.mark(1)
    ms = ctx.elapsed_ms(0, 1)
    torch.cuda.synchronize()
    clk = clocks.stop() if clocks else None
    sol.loop_end()
    _barrier(world)
    ms_max, value = replica_throughput(cfg.cells, args.steps, ms, world)

    # ---- roofline: per-kernel-class device time over a few further steps
    ctx.kernel_timing(True)
    nprof = max(2, min(args.steps, 4))
    sol.step(nprof)
    kt = ctx.kernel_times()
    ctx.kernel_timing(False)
    cls = max((k for k in kt if kt[k][1] > 0), key=lambda k: kt[k][0])
    avg_ms = kt[cls][0] / kt[cls][1]
    own_bytes_launch = kernel_bytes_per_cell(cls, esz) * cfg.cells
    bytes_launch = (STEP_BYTES_PER_CELL * esz / 8 / 4 * cfg.cells) if cls in STAGE_KERNELS else own_bytes_launch
    peak, peak_kind = _peaks()
    achieved = bytes_launch / (avg_ms / 1e3) / 1e9
    traffic = _traffic_table().get((cls, args.workload, args.precision))
    step_ms = ms_max / args.steps
    roofline = {"bound": "hbm", "kernel": cls, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": peak_kind,
                "traffic": (traffic * cfg.cells if traffic is not None else None),
                "algorithmic_bytes_per_launch": bytes_launch, "avg_launch_ms": avg_ms,
                "kernel_own_bytes_per_launch": own_bytes_launch,
                "kernel_own_gbs": own_bytes_launch / (avg_ms / 1e3) / 1e9,
                "kernel_ms_per_step": {k: v[0] / nprof for k, v in kt.items()},
                "kernel_share": {k: (v[0] / max(sum(x[0] for x in kt.values()), 1e-30)) for k, v in kt.items()},
                "step_achieved_gbs": STEP_BYTES_PER_CELL * esz / 8 * cfg.cells / (step_ms / 1e3) / 1e9,
                "step_frac": STEP_BYTES_PER_CELL * esz / 8 * cfg.cells / (step_ms / 1e3) / 1e9 / peak}

    # ---- e2e through the public solver API with host buffers (pinned): the state is
    # uploaded, K steps run on the device loop with every step's history (dt, |u|max, the
    # probe lines, monitor rows) read back, and the final state downloaded -- all timed
    st = sol.state()
    pinned = {k: torch.empty(v.shape, dtype=torch.float64, pin_memory=True) for k, v in st.items()}
    for k, v in st.items():
        pinned[k].numpy()[...] = v
    host_state = {k: t.numpy() for k, t in pinned.items()}
    pinned_out = {k: torch.empty(v.shape, dtype=torch.float64, pin_memory=True).numpy() for k, v in st.items()}
    tmpd = tempfile.mkdtemp(prefix="lesbench_")
    sol.set_outputs(tmpd, N.LES_OUT_PROBES | N.LES_OUT_MONITOR)
    sol.loop_begin(chunk=args.steps)
    _barrier(world)
    ctx.sync()
    ctx.mark(2)
    ctx.upload_state(host_state)
    sol.loop_run(args.steps)
    out = ctx.download_state(out=pinned_out)
    ctx.mark(3)
    sol.loop_end()
    e2e_ms = _max_over_ranks(ctx.elapsed_ms(2, 3), world)
    e2e_value = world * cfg.cells * args.steps / (e2e_ms / 1e3)
    sol.set_outputs(None, 0)
    shutil.rmtree(tmpd, ignore_errors=True)
    stations = [int(x / (cfg.lx / cfg.nx)) for x in (0.010, 0.015, 0.020, 0.025, 0.030, 0.035, 0.040)]
    stations = [i for i in stations if 0 < i < cfg.nx - 1]
    state_bytes = 11 * cfg.cells * 8
    h2d = state_bytes / args.steps
    d2h = state_bytes / args.steps + 8 * (2 + 6) + len(stations) * cfg.ny * 6 * 8
    del out

    # ---- the literal host-driven ABI cycle per step (dt inputs -> host rand() ->
    # lesgpu_set_inflow -> lesgpu_step -> probe lines), for comparison
    nh = max(2, min(args.steps, 10))
    ctx.mark(4)
    for _ in range(nh):
        sol.step(1)
        ctx.probe_lines(stations, cfg.nz // 2)
    ctx.mark(5)
    host_ms = ctx.elapsed_ms(4, 5) / nh
    n_inlet = int((sol.attribute()[0] == 1).sum())

    result = None
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            r = cpu_reference_rate(args.workload, REF_SAMPLE_STEPS, budget_s=REF_SAMPLE_BUDGET_S,
                                   threads=os.cpu_count() or 1)
            if r is not None:
                rate, n, cores, kind, sample = r
                cpu = {"value": rate, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample}
        result = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if prec == N.FP64 else "f32",
            "data": "synthetic: the reference's initial flame state, seeded SEM inflow, placeholder species properties",
            "config": {"workload": WORKLOADS.get(args.workload, args.workload), "grid": [cfg.nx, cfg.ny, cfg.nz],
                       "cells": cfg.cells, "precision": args.precision, "parallelism": f"replicas x{world}",
                       "l2": f"inputs larger than L2 ({ctx.device_bytes / 2**30:.2f} GiB resident per replica)",
                       "tiles": tiles},
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "path": "les_solver: upload state, device loop with per-step history read-back, download"},
            "host_driven_step": {"ms_per_step": host_ms, "value": world * cfg.cells / (host_ms / 1e3),
                                 "h2d_bytes_per_step": cfg.num_vortices * 7 * 8 + n_inlet * 3 * 8 + 16,
                                 "d2h_bytes_per_step": 24 + len(stations) * cfg.ny * 6 * 8},
            "gpu_launches": per_step_launches * args.steps,
            "clocks": clk,
        }
        print(json.dumps(result))
    sol.close()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="c2")
    ap.add_argument("--precision", choices=["fp64", "fp32"], default="fp64")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--tiles", choices=["auto", "default"], default="auto",
                    help="auto: per-class thread-block tiles picked by lesgpu_autotune; default: 32x8 everywhere")
    args = ap.parse_args(argv)
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference_arm(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
