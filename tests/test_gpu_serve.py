"""Serving loop on the GPU: a request's result is the same alone and in a mix of other
requests arriving while it runs (bit-identical: each request has its own state, rand()
stream and tiles, and the device loop does not depend on chunking), whether requests are set
up by the stepping thread or by the server's workers; admission never exceeds the HBM
budget, and cancellation frees the request's memory."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STATE = ["u", "v", "w", "T", "G", "rho", "Y0", "Y1", "Y2", "Y3", "Y4"]


@pytest.fixture(scope="module")
def N(lesgpu_native, cuda_device):
    return lesgpu_native


@pytest.fixture(scope="module")
def S(N):
    from lesgpu import serve
    return serve


def _same(a, b, what):
    for f in STATE:
        np.testing.assert_array_equal(a[f], b[f], err_msg=f"{what}: {f}")


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_result_same_alone_and_in_the_mix(N, S, prec):
    from lesgpu.config import preset
    P = N.FP32 if prec == "fp32" else N.FP64
    target = preset("small", seed=91, cs_unburned=0.12, relax=3000.0)
    # alone: set-up on the stepping thread; in the mix: on the server's worker threads
    alone = S.Server(quantum=7, prep_threads=0)
    rid = alone.submit(target, 23, P)
    alone.drain()
    assert alone.info(rid)["state_name"] == "done"
    r_alone = alone.result(rid)
    alone.close()

    mix = S.Server(quantum=5, max_slots=3, prep_threads=3)
    others = [mix.submit(preset("tiny", seed=5), 40, P), mix.submit(preset("c1", seed=6, accel_strength=1.0), 12, P)]
    mix.step()
    mix.step()
    rid = mix.submit(target, 23, P)                       # arrives while others run
    others.append(mix.submit(preset("tiny", seed=8), 9, P))
    mix.step()
    others.append(mix.submit(preset("small", seed=9), 30, P))
    mix.drain()
    for o in others + [rid]:
        assert mix.info(o)["state_name"] == "done", mix.info(o)
    _same(mix.result(rid), r_alone, "alone vs mix")
    st = mix.stats()
    assert st["done"] == 5 and st["active"] == 0 and st["bytes_in_use"] == 0
    assert st["latency_p99_s"] >= st["latency_p50_s"] > 0 and st["cell_steps_per_s"] > 0
    mix.close()

    solo = N.Solver(target, precision=P)
    solo.run_device(23, chunk=23)
    _same(solo.state(), r_alone, "server vs les_solver")
    solo.close()


def test_budget_bounds_admission(N, S):
    from lesgpu.config import preset
    cfgs = [preset("c1", seed=s) for s in range(4)]
    one = S.request_bytes(cfgs[0], N.FP32, 4)
    srv = S.Server(budget_bytes=int(one * 2.5), quantum=4)
    ids = [srv.submit(c, 10, N.FP32) for c in cfgs]
    seen_active = 0
    while True:
        left = srv.step()
        st = srv.stats()
        assert st["bytes_in_use"] <= int(one * 2.5)
        assert st["active"] <= 2
        seen_active = max(seen_active, st["active"])
        for i in ids:
            inf = srv.info(i)
            if inf["state_name"] == "active":
                assert 0 < inf["device_bytes"] <= inf["bytes"]
        if left == 0:
            break
    assert seen_active == 2
    assert all(srv.info(i)["state_name"] == "done" for i in ids)
    srv.close()


def test_cancel_active_request_frees_memory(N, S):
    from lesgpu.config import preset
    srv = S.Server(quantum=3)
    a = srv.submit(preset("c1", seed=1), 30, N.FP32)
    b = srv.submit(preset("tiny", seed=2), 6, N.FP32)
    srv.step()
    assert srv.info(a)["state_name"] == "active"
    before = srv.stats()["bytes_in_use"]
    srv.cancel(a)
    assert srv.stats()["bytes_in_use"] == before - srv.info(a)["bytes"]
    srv.drain()
    assert srv.info(a)["state_name"] == "cancelled" and srv.info(b)["state_name"] == "done"
    with pytest.raises(N.LesgpuError):
        srv.result(a)
    srv.close()


def test_poisson_replay_small(N, S):
    """A short replay of the serving workload shape (small grids, few steps)."""
    reqs = S.poisson_requests(12, rate=50.0, steps=(5, 15), seed=1, grids=("tiny", "small", "c1"))
    srv = S.Server(quantum=4, autotune=True)
    st = srv.replay(reqs) if hasattr(srv, "replay") else S.replay(srv, reqs, N.FP32)
    assert st["done"] == 12 and st["failed"] == 0
    assert st["latency_p99_s"] >= st["latency_p50_s"] > 0
    srv.close()


def test_served_request_statistics_without_probe_files(N, S, tmp_path):
    """A request with LES_OUT_PSTAT alone: no probe files, and profile_stats.bin at the end
    holds the device-accumulated statistics of its rows -- the same as les_solver's own
    device statistics of the same run (summed in other chunks: counts exact, sums 1e-12)."""
    from lesgpu import stats
    from lesgpu.config import preset
    cfg = preset("c1", seed=31)
    srv = S.Server(quantum=9, prep_threads=2)
    rid = srv.submit(cfg, 60, N.FP64, out_dir=str(tmp_path), out_flags=N.LES_OUT_PSTAT)
    srv.submit(preset("tiny", seed=3), 25, N.FP64)
    srv.drain()
    assert srv.info(rid)["state_name"] == "done"
    srv.close()
    assert not list(tmp_path.glob("probe_data_*"))
    edges, sums = stats.read_moments_file(str(tmp_path / "profile_stats.bin"))
    solo = N.Solver(cfg)
    e2 = solo.pstat_begin()
    solo.run_device(60, chunk=64)
    ref = solo.pstat_read()
    solo.close()
    for k in e2:
        np.testing.assert_array_equal(edges[k], e2[k])
    got, want = stats.from_moments(sums, edges), stats.from_moments(ref, e2)
    assert sums[0] == ref[0] > 1000
    np.testing.assert_allclose(sums, ref, rtol=1e-12, atol=1e-9)
    np.testing.assert_allclose(got["flame_profile"]["re_uv"], want["flame_profile"]["re_uv"], rtol=1e-9, atol=1e-14)
