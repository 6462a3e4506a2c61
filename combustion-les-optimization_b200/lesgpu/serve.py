"""Serving loop (les_serve_* of include/les_serve.h): many solve requests on one GPU.

``Server`` wraps the C request loop; ``poisson_requests`` draws the serving workload
(Poisson arrivals at a mean rate, grids uniform over 64x32x32, 128x64x64, 192x96x96 and
256x128x128, step counts uniform over an integer range, model constants drawn as for the
batched ensemble); ``replay`` submits the requests at their arrival times while stepping the
server and returns the latency / throughput summary.

Measurement (one JSON line):

    python -m lesgpu.serve --requests 100 --rate 20 --steps 50 200 --quantum 16
"""
from __future__ import annotations

import ctypes as C
import json
import time
from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import native as N
from .config import PRESETS, SolverConfig

QUEUED, ACTIVE, DONE, CANCELLED, FAILED = 0, 1, 2, 3, 4
STATE_NAMES = {QUEUED: "queued", ACTIVE: "active", DONE: "done", CANCELLED: "cancelled", FAILED: "failed"}


class ServeOptions(C.Structure):
    _fields_ = [("budget_bytes", C.c_size_t), ("max_slots", C.c_int), ("quantum_steps", C.c_int),
                ("keep_results", C.c_int), ("autotune", C.c_int), ("backfill", C.c_int), ("device", C.c_int),
                ("chem_path", C.c_char * 1024), ("tran_path", C.c_char * 1024), ("prep_threads", C.c_int),
                ("policy", C.c_int)]


# admission order (les_serve.h)
FIFO, SHORTEST = 0, 1


class RequestInfo(C.Structure):
    _fields_ = [("state", C.c_int), ("error", C.c_int), ("steps_done", C.c_int), ("nsteps", C.c_int),
                ("bytes", C.c_size_t), ("device_bytes", C.c_size_t), ("t_submit", C.c_double),
                ("t_admit", C.c_double), ("t_done", C.c_double), ("latency_s", C.c_double)]


class Summary(C.Structure):
    _fields_ = [("submitted", C.c_longlong), ("queued", C.c_longlong), ("active", C.c_longlong),
                ("done", C.c_longlong), ("failed", C.c_longlong), ("cancelled", C.c_longlong),
                ("bytes_in_use", C.c_size_t), ("cell_steps", C.c_double), ("busy_s", C.c_double),
                ("cell_steps_per_s", C.c_double), ("latency_p50_s", C.c_double), ("latency_p99_s", C.c_double),
                ("latency_max_s", C.c_double)]


def _lib():
    L = N.lib()
    if getattr(L, "_serve_sigs", False):
        return L
    vp = C.c_void_p
    N._sig(L, "les_serve_default_options", None, [C.POINTER(ServeOptions)])
    N._sig(L, "les_serve_request_bytes", C.c_size_t, [C.POINTER(N.LesgpuConfig), C.c_int])
    N._sig(L, "les_serve_create", C.c_int, [C.POINTER(ServeOptions), C.POINTER(vp)])
    N._sig(L, "les_serve_submit", C.c_int, [vp, C.POINTER(N.LesgpuConfig), C.c_int, C.c_char_p, C.c_int,
                                            C.POINTER(C.c_longlong)])
    N._sig(L, "les_serve_step", C.c_int, [vp])
    N._sig(L, "les_serve_cancel", C.c_int, [vp, C.c_longlong])
    N._sig(L, "les_serve_info", C.c_int, [vp, C.c_longlong, C.POINTER(RequestInfo)])
    N._sig(L, "les_serve_result", C.c_int, [vp, C.c_longlong, C.POINTER(C.c_void_p), C.c_int])
    N._sig(L, "les_serve_release", C.c_int, [vp, C.c_longlong])
    N._sig(L, "les_serve_stats", C.c_int, [vp, C.POINTER(Summary)])
    N._sig(L, "les_serve_last_error", C.c_char_p, [vp])
    N._sig(L, "les_serve_destroy", None, [vp])
    L._serve_sigs = True
    return L


def request_bytes(cfg: SolverConfig, precision: int = N.FP32, quantum: int = 16) -> int:
    c = N.LesgpuConfig.from_config(cfg, precision, 0)
    return int(_lib().les_serve_request_bytes(C.byref(c), quantum))


class Server:
    def __init__(self, budget_bytes: int = 150 * 10**9, max_slots: int = 16, quantum: int = 16,
                 keep_results: bool = True, autotune: bool = False, backfill: bool = False, device: int = 0,
                 chem: str = N.CHEM_BIN, tran: str = N.TRAN_BIN, prep_threads: Optional[int] = None,
                 policy: int = FIFO):
        L = _lib()
        o = ServeOptions()
        L.les_serve_default_options(C.byref(o))
        o.budget_bytes, o.max_slots, o.quantum_steps = int(budget_bytes), max_slots, quantum
        o.keep_results, o.autotune, o.backfill, o.device = int(keep_results), int(autotune), int(backfill), device
        o.chem_path, o.tran_path = chem.encode(), tran.encode()
        if prep_threads is not None:
            o.prep_threads = prep_threads
        o.policy = policy
        h = C.c_void_p()
        rc = L.les_serve_create(C.byref(o), C.byref(h))
        if rc:
            raise N.LesgpuError(rc, "les_serve_create failed")
        self._h = h
        self.device = device
        self.quantum = quantum
        self.cfgs: Dict[int, SolverConfig] = {}

    def _check(self, rc, what):
        if rc < 0:
            raise N.LesgpuError(rc, f"{what}: {_lib().les_serve_last_error(self._h).decode()}")
        return rc

    def submit(self, cfg: SolverConfig, nsteps: int, precision: int = N.FP32, out_dir: Optional[str] = None,
               out_flags: int = 0) -> int:
        c = N.LesgpuConfig.from_config(cfg, precision, self.device)
        rid = C.c_longlong(-1)
        self._check(_lib().les_serve_submit(self._h, C.byref(c), nsteps, out_dir.encode() if out_dir else None,
                                            out_flags, C.byref(rid)), "submit")
        self.cfgs[rid.value] = cfg
        return rid.value

    def step(self) -> int:
        return self._check(_lib().les_serve_step(self._h), "step")

    def drain(self):
        while self.step() > 0:
            pass

    def cancel(self, rid: int):
        self._check(_lib().les_serve_cancel(self._h, rid), "cancel")

    def info(self, rid: int) -> dict:
        i = RequestInfo()
        self._check(_lib().les_serve_info(self._h, rid, C.byref(i)), "info")
        d = {k: getattr(i, k) for k, _ in RequestInfo._fields_}
        d["state_name"] = STATE_NAMES.get(i.state, "?")
        return d

    def result(self, rid: int) -> Dict[str, np.ndarray]:
        cfg = self.cfgs[rid]
        shape = (cfg.nx, cfg.ny, cfg.nz)
        out = {f: np.empty(shape) for f in N.STATE_NAMES}
        ptrs = (C.c_void_p * len(N.STATE_NAMES))(*[out[f].ctypes.data for f in N.STATE_NAMES])
        self._check(_lib().les_serve_result(self._h, rid, ptrs, len(N.STATE_NAMES)), "result")
        return out

    def release(self, rid: int):
        self._check(_lib().les_serve_release(self._h, rid), "release")

    def stats(self) -> dict:
        s = Summary()
        self._check(_lib().les_serve_stats(self._h, C.byref(s)), "stats")
        return {k: getattr(s, k) for k, _ in Summary._fields_}

    def close(self):
        if getattr(self, "_h", None):
            _lib().les_serve_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


SERVE_GRIDS = ("c1", "e128", "s192", "c2")     # 64x32x32, 128x64x64, 192x96x96, 256x128x128


@dataclass
class Request:
    t_arrival: float
    cfg: SolverConfig
    nsteps: int


def poisson_requests(n: int = 1000, rate: float = 20.0, steps=(500, 2000), seed: int = 2024,
                     grids: Sequence[str] = SERVE_GRIDS) -> List[Request]:
    """Seeded Poisson arrivals (exponential gaps at ``rate``/s); grid uniform over ``grids``;
    step count uniform over steps[0]..steps[1] inclusive; CS_UNBURNED, flame-acceleration
    strength and nudging drawn as for the batched ensemble."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n))
    g = rng.integers(0, len(grids), n)
    ns = rng.integers(steps[0], steps[1] + 1, n)
    cs = rng.uniform(0.08, 0.22, n)
    d = SolverConfig()
    strength = rng.uniform(0.0, 2.0, n) * d.accel_strength
    relax = rng.uniform(0.0, 1.0, n) * d.relax
    return [Request(float(t[q]), PRESETS[grids[g[q]]].replace(cs_unburned=float(cs[q]), accel_strength=float(strength[q]),
                                                             relax=float(relax[q]), seed=int(seed + 31 * q + 7)),
                    int(ns[q])) for q in range(n)]


def replay(server: Server, requests: Sequence[Request], precision: int = N.FP32, time_scale: float = 1.0,
           keep: bool = False) -> dict:
    """Submit each request at its arrival time (scaled by ``time_scale``) while stepping the
    server; returns the server's summary plus the request ids."""
    t0 = time.monotonic()
    ids = []
    q = 0
    pending = 0
    while q < len(requests) or pending > 0:
        now = time.monotonic() - t0
        while q < len(requests) and requests[q].t_arrival * time_scale <= now:
            ids.append(server.submit(requests[q].cfg, requests[q].nsteps, precision))
            q += 1
        pending = server.step()
        if pending == 0 and q < len(requests):
            time.sleep(max(0.0, min(0.01, requests[q].t_arrival * time_scale - (time.monotonic() - t0))))
    s = server.stats()
    s["ids"] = ids
    s["wall_s"] = time.monotonic() - t0
    if not keep:
        for rid in ids:
            server.release(rid)
    return s


def main(argv=None) -> int:
    import argparse
    ap = argparse.ArgumentParser(description="Replay a seeded Poisson request stream through the serving loop")
    ap.add_argument("--requests", type=int, default=100)
    ap.add_argument("--rate", type=float, default=20.0, help="mean arrivals per second")
    ap.add_argument("--steps", type=int, nargs=2, default=(50, 200), metavar=("MIN", "MAX"))
    ap.add_argument("--quantum", type=int, default=16)
    ap.add_argument("--precision", choices=["fp64", "fp32"], default="fp32")
    ap.add_argument("--budget-gb", type=float, default=150.0)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--prep-threads", type=int, default=None, help="set-up / tear-down worker threads")
    ap.add_argument("--max-slots", type=int, default=16, help="at most this many requests on the device at once")
    ap.add_argument("--policy", choices=["fifo", "shortest"], default="fifo",
                    help="admission order: arrival, or least work (cells x steps) first")
    a = ap.parse_args(argv)
    prec = N.FP32 if a.precision == "fp32" else N.FP64
    reqs = poisson_requests(a.requests, rate=a.rate, steps=tuple(a.steps), seed=a.seed)
    srv = Server(budget_bytes=int(a.budget_gb * 1e9), max_slots=a.max_slots, quantum=a.quantum, autotune=True,
                 prep_threads=a.prep_threads, policy=SHORTEST if a.policy == "shortest" else FIFO)
    st = replay(srv, reqs, prec)
    srv.close()
    st.pop("ids")
    st.update(requests=a.requests, rate=a.rate, steps=list(a.steps), quantum=a.quantum, precision=a.precision,
              prep_threads=a.prep_threads, max_slots=a.max_slots, policy=a.policy,
              demand_cell_steps=sum(r.cfg.cells * r.nsteps for r in reqs))
    print(json.dumps(st))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
