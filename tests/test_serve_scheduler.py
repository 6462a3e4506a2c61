"""The serving scheduler (host/les_serve.c) with its worker threads, on the CPU.

The scheduler is compiled here against a stand-in for the solver and device library
(tests/serve_fake/fake_backend.c): "device memory" is a counter with an optional limit,
set-up and stepping take a little wall time, and the downloaded final state encodes the
request's seed, the steps it ran and its tiles.  The tests check what the GPU tests cannot
force: the budget is never exceeded while set-ups run on several threads, a set-up that finds
the device full is retried until it fits, a request cancelled during its set-up returns its
memory, every request runs exactly its steps, tiles are tuned once per grid shape, and the
results do not depend on whether the stepping thread or the workers do the set-up.
"""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT

PKG = os.path.join(ROOT, "combustion-les-optimization_b200")


@pytest.fixture(scope="module")
def fake(tmp_path_factory, lesgpu_native):
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("gcc not available")
    out = str(tmp_path_factory.mktemp("fakeserve") / "libfakeserve.so")
    subprocess.run([gcc, "-shared", "-fPIC", "-O1", "-std=c11", "-pthread", "-I", os.path.join(ROOT, "include"),
                    "-I", os.path.join(PKG, "host"), os.path.join(PKG, "host", "les_serve.c"),
                    os.path.join(ROOT, "tests", "serve_fake", "fake_backend.c"), "-o", out], check=True)
    from lesgpu import serve as S
    L = C.CDLL(out)
    vp = C.c_void_p
    L.les_serve_default_options.argtypes = [C.POINTER(S.ServeOptions)]
    L.les_serve_create.argtypes = [C.POINTER(S.ServeOptions), C.POINTER(vp)]
    L.les_serve_submit.argtypes = [vp, C.c_void_p, C.c_int, C.c_char_p, C.c_int, C.POINTER(C.c_longlong)]
    L.les_serve_step.argtypes = [vp]
    L.les_serve_cancel.argtypes = [vp, C.c_longlong]
    L.les_serve_info.argtypes = [vp, C.c_longlong, C.POINTER(S.RequestInfo)]
    L.les_serve_result.argtypes = [vp, C.c_longlong, C.POINTER(C.c_void_p), C.c_int]
    L.les_serve_stats.argtypes = [vp, C.POINTER(S.Summary)]
    L.les_serve_request_bytes.argtypes = [C.c_void_p, C.c_int]
    L.les_serve_request_bytes.restype = C.c_size_t
    L.les_serve_destroy.argtypes = [vp]
    L.fake_configure.argtypes = [C.c_size_t, C.c_double, C.c_double]
    L.fake_stats.argtypes = [C.POINTER(C.c_longlong)]
    L.fake_fail_tunes.argtypes = [C.c_int]
    return L, S, lesgpu_native


def _cfg(N, nx, ny, nz, seed):
    from lesgpu.config import preset
    return N.LesgpuConfig.from_config(preset("tiny").replace(nx=nx, ny=ny, nz=nz, seed=seed), N.FP32, 0)


class Server:
    def __init__(self, fake, budget, slots=8, quantum=4, threads=4, autotune=True, policy=0, backfill=0):
        L, S, N = fake
        self.L, self.S, self.N = L, S, N
        o = S.ServeOptions()
        L.les_serve_default_options(C.byref(o))
        o.budget_bytes, o.max_slots, o.quantum_steps, o.autotune, o.prep_threads = budget, slots, quantum, int(autotune), threads
        o.policy, o.backfill = policy, backfill
        o.chem_path, o.tran_path = b"unused", b"unused"
        self.h = C.c_void_p()
        assert L.les_serve_create(C.byref(o), C.byref(self.h)) == 0
        self.cfgs = {}

    def submit(self, cfg, nsteps):
        rid = C.c_longlong(-1)
        rc = self.L.les_serve_submit(self.h, C.byref(cfg), nsteps, None, 0, C.byref(rid))
        assert rc == 0, rc
        self.cfgs[rid.value] = cfg
        return rid.value

    def step(self):
        r = self.L.les_serve_step(self.h)
        assert r >= 0, r
        return r

    def stats(self):
        s = self.S.Summary()
        assert self.L.les_serve_stats(self.h, C.byref(s)) == 0
        return {k: getattr(s, k) for k, _ in self.S.Summary._fields_}

    def info(self, rid):
        i = self.S.RequestInfo()
        assert self.L.les_serve_info(self.h, rid, C.byref(i)) == 0
        return {k: getattr(i, k) for k, _ in self.S.RequestInfo._fields_}

    def result(self, rid):
        c = self.cfgs[rid]
        n = c.nx * c.ny * c.nz
        arrs = [np.empty(n) for _ in range(11)]
        ptrs = (C.c_void_p * 11)(*[a.ctypes.data for a in arrs])
        assert self.L.les_serve_result(self.h, rid, ptrs, 11) == 0
        return arrs

    def fake_stats(self):
        out = (C.c_longlong * 8)()
        self.L.fake_stats(out)
        return dict(zip(["used", "peak", "creates", "enomem", "tunes", "live", "max_live", "collect_errors"], out))

    def close(self):
        self.L.les_serve_destroy(self.h)


SHAPES = [(8, 4, 4), (12, 6, 4), (16, 4, 8), (8, 4, 4), (20, 8, 4), (12, 6, 4)]


def _requests(fake, n):
    _, _, N = fake
    return [(_cfg(N, *SHAPES[q % len(SHAPES)], seed=100 + q), 5 + (7 * q) % 23) for q in range(n)]


def _drain(srv, check=None):
    while True:
        left = srv.step()
        if check:
            check()
        if left == 0:
            return


def test_budget_slots_and_steps_with_worker_threads(fake):
    L, S, N = fake
    L.fake_configure(0, 0.003, 200.0)
    reqs = _requests(fake, 24)
    one = max(L.les_serve_request_bytes(C.byref(c), 4) for c, _ in reqs)
    budget = int(2.5 * one)
    srv = Server(fake, budget, slots=8, quantum=4, threads=4)
    ids = [srv.submit(c, n) for c, n in reqs]
    seen = {"active": 0}

    def check():
        st = srv.stats()
        assert st["bytes_in_use"] <= budget
        assert srv.fake_stats()["used"] <= budget
        seen["active"] = max(seen["active"], st["active"])

    _drain(srv, check)
    st = srv.stats()
    assert st["done"] == 24 and st["failed"] == 0 and st["bytes_in_use"] == 0
    assert seen["active"] >= 2
    fs = srv.fake_stats()
    assert fs["collect_errors"] == 0 and fs["live"] == 0 and fs["creates"] == 24
    assert fs["tunes"] == len(set(SHAPES))                 # one tuning per grid shape
    for rid, (c, n) in zip(ids, reqs):
        r = srv.result(rid)
        for k in range(11):
            assert np.all(r[k] == c.seed * 1000 + n + k + 1e6 * (c.nx % 8)), (rid, k)
    srv.close()


@pytest.mark.parametrize("threads", [0, 3])
def test_failed_autotune_is_retried_not_cached(fake, threads):
    """The first autotune of a shape fails: that request fails, the next request of the same
    shape tunes again, and every later one gets the published tiles (no request runs its own
    tuning or keeps the failure)."""
    L, S, N = fake
    L.fake_configure(0, 0.002, 100.0)
    L.fake_fail_tunes(1)
    srv = Server(fake, 10 ** 12, slots=4, quantum=3, threads=threads)
    reqs = [(_cfg(N, 12, 6, 4, 300 + q), 4 + q) for q in range(8)]
    ids = [srv.submit(c, n) for c, n in reqs]
    _drain(srv)
    st = srv.stats()
    fs = srv.fake_stats()
    assert st["failed"] == 1 and st["done"] == 7, st
    assert fs["tunes"] == 2 and fs["live"] == 0, fs
    failed = [r for r in ids if srv.info(r)["error"] != 0]
    assert len(failed) == 1
    for rid, (c, n) in zip(ids, reqs):
        if rid in failed:
            continue
        assert srv.result(rid)[0][0] == c.seed * 1000 + n + 1e6 * (c.nx % 8)
    srv.close()


def test_full_device_retries_the_set_up(fake):
    L, S, N = fake
    reqs = _requests(fake, 10)
    sizes = [L.les_serve_request_bytes(C.byref(c), 4) for c, _ in reqs]
    # the budget admits about three requests, the device holds only a little more than one
    L.fake_configure(int(1.2 * max(sizes)), 0.002, 500.0)
    srv = Server(fake, int(3.2 * max(sizes)), slots=8, quantum=4, threads=3)
    ids = [srv.submit(c, n) for c, n in reqs]
    _drain(srv)
    st = srv.stats()
    fs = srv.fake_stats()
    assert st["done"] == 10 and st["failed"] == 0
    assert fs["enomem"] > 0 and fs["live"] == 0
    for rid, (c, n) in zip(ids, reqs):
        assert srv.result(rid)[0][0] == c.seed * 1000 + n + 1e6 * (c.nx % 8)
    srv.close()


def test_cancel_during_set_up_returns_the_memory(fake):
    L, S, N = fake
    L.fake_configure(0, 0.6, 50.0)                         # slow set-up
    srv = Server(fake, 10 ** 12, slots=4, quantum=2, threads=2)
    a = srv.submit(_cfg(N, 16, 8, 8, 1), 400)
    srv.step()                                             # nothing ran: waits for a's set-up
    assert srv.info(a)["state"] == 1
    b = srv.submit(_cfg(N, 8, 4, 4, 2), 10)
    srv.step()                                             # b goes to a worker; a steps
    assert srv.info(b)["state"] == 0                       # still queued (being set up)
    before = srv.stats()["bytes_in_use"]
    assert L.les_serve_cancel(srv.h, b) == 0
    assert srv.info(b)["state"] == 3
    assert srv.stats()["bytes_in_use"] == before - srv.info(b)["bytes"]
    assert L.les_serve_cancel(srv.h, a) == 0              # active, with a quantum in flight
    assert srv.info(a)["state"] == 3
    assert srv.stats()["bytes_in_use"] == 0
    assert srv.step() == 0
    fs = srv.fake_stats()
    assert fs["live"] == 0 and fs["collect_errors"] == 0
    srv.close()


def test_results_do_not_depend_on_who_does_the_set_up(fake):
    L, S, N = fake
    out = []
    for threads in (0, 4):
        L.fake_configure(0, 0.001, 100.0)
        reqs = _requests(fake, 12)
        one = max(L.les_serve_request_bytes(C.byref(c), 3) for c, _ in reqs)
        srv = Server(fake, int(4.5 * one), slots=3, quantum=3, threads=threads)
        ids = [srv.submit(c, n) for c, n in reqs]
        _drain(srv)
        assert srv.stats()["done"] == 12
        out.append([srv.result(r)[3][0] for r in ids])
        srv.close()
    assert out[0] == out[1]


@pytest.mark.parametrize("threads,limit_factor", [(1, 0), (2, 1.5), (8, 2.2)])
def test_stress_many_requests(fake, threads, limit_factor):
    """Sixty requests arriving while others run, a tight budget and (for two of the cases) a
    device that holds fewer requests than the budget admits: every request finishes with
    exactly its steps and nothing is left allocated."""
    L, S, N = fake
    rng = np.random.default_rng(threads)
    reqs = [(_cfg(N, *SHAPES[int(rng.integers(len(SHAPES)))], seed=500 + q), int(rng.integers(1, 40)))
            for q in range(60)]
    one = max(L.les_serve_request_bytes(C.byref(c), 5) for c, _ in reqs)
    L.fake_configure(int(limit_factor * one), 0.0005, 300.0)
    srv = Server(fake, int(3.5 * one), slots=6, quantum=5, threads=threads)
    ids = []
    q = 0
    while True:
        for _ in range(int(rng.integers(0, 4))):            # a few arrivals per round
            if q < len(reqs):
                ids.append(srv.submit(*reqs[q]))
                q += 1
        left = srv.step()
        assert srv.stats()["bytes_in_use"] <= int(3.5 * one)
        if left == 0 and q == len(reqs):
            break
    assert srv.stats()["done"] == 60 and srv.stats()["failed"] == 0
    fs = srv.fake_stats()
    assert fs["live"] == 0 and fs["used"] == 0 and fs["collect_errors"] == 0
    for rid, (c, n) in zip(ids, reqs):
        assert srv.result(rid)[5][0] == c.seed * 1000 + n + 5 + 1e6 * (c.nx % 8)
    srv.close()


@pytest.mark.parametrize("threads,backfill", [(0, 0), (3, 0), (3, 1)])
def test_shortest_work_first_admission(fake, threads, backfill):
    """LES_SERVE_SHORTEST admits the queued request with the least work (cells x steps)
    first: with one slot, requests submitted together complete in order of work (ties in
    arrival order), every request finishes with its steps, and the budget is never exceeded."""
    L, S, N = fake
    L.fake_configure(0, 0.001, 50.0)
    # requests 2 and 5 ask for the same work (2560 cell-steps): 2 arrived first, so it goes first
    shapes = [(20, 8, 4), (8, 4, 4), (16, 4, 8), (12, 6, 4), (8, 4, 4), (8, 8, 8)]
    steps = [30, 40, 5, 12, 9, 5]
    reqs = [(_cfg(N, *shapes[q], seed=700 + q), steps[q]) for q in range(len(shapes))]
    one = max(L.les_serve_request_bytes(C.byref(c), 3) for c, _ in reqs)
    srv = Server(fake, int(2.5 * one), slots=1, quantum=3, threads=threads, policy=S.SHORTEST, backfill=backfill)
    ids = [srv.submit(c, n) for c, n in reqs]
    order = []
    while True:
        left = srv.step()
        assert srv.stats()["bytes_in_use"] <= int(2.5 * one)
        for rid in ids:
            if rid not in order and srv.info(rid)["state"] == 2:          # LES_REQ_DONE
                order.append(rid)
        if left == 0:
            break
    work = {rid: c.nx * c.ny * c.nz * n for rid, (c, n) in zip(ids, reqs)}
    assert len(set(work.values())) < len(work)           # the tie is there
    assert sorted(order, key=lambda r: (work[r], r)) == order, (order, work)
    for rid, (c, n) in zip(ids, reqs):
        assert srv.result(rid)[0][0] == c.seed * 1000 + n + 1e6 * (c.nx % 8)
    srv.close()


def test_unknown_policy_is_refused(fake):
    L, S, N = fake
    o = S.ServeOptions()
    L.les_serve_default_options(C.byref(o))
    o.chem_path, o.tran_path, o.policy = b"unused", b"unused", 7
    h = C.c_void_p()
    assert L.les_serve_create(C.byref(o), C.byref(h)) == -1
