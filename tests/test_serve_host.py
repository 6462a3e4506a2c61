"""Serving loop host logic on the CPU: admission budget arithmetic, refusal of requests
that can never fit, queue bookkeeping, cancellation and the Poisson workload generator.
No call here touches a GPU (les_serve_create / submit / cancel / stats are host-only)."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def S(lesgpu_native):
    from lesgpu import serve
    return serve


def test_request_bytes_grow_with_grid_and_precision(S, lesgpu_native):
    from lesgpu.config import preset
    N = lesgpu_native
    b = [S.request_bytes(preset(g), N.FP32) for g in ("c1", "e128", "s192", "c2")]
    assert b == sorted(b) and b[0] > 0
    c2 = preset("c2")
    # at least the 59 per-cell fields: all 8-byte in the FP64 form; in the FP32 form the 11
    # state fields stay 8-byte and the other 48 are 4-byte
    assert S.request_bytes(c2, N.FP64) >= 59 * 8 * c2.cells
    assert S.request_bytes(c2, N.FP32) >= (11 * 8 + 48 * 4) * c2.cells
    assert S.request_bytes(c2, N.FP64) > 1.6 * S.request_bytes(c2, N.FP32)


def test_submit_refuses_what_never_fits_and_queues_the_rest(S, lesgpu_native):
    from lesgpu.config import preset
    N = lesgpu_native
    need = S.request_bytes(preset("e128"), N.FP32)
    srv = S.Server(budget_bytes=need + 1000)
    with pytest.raises(N.LesgpuError) as e:
        srv.submit(preset("c2"), 10)
    assert e.value.code == N.LESGPU_ENOMEM
    a = srv.submit(preset("e128"), 10)
    b = srv.submit(preset("c1"), 5)
    assert (a, b) == (0, 1)
    st = srv.stats()
    assert st["submitted"] == 2 and st["queued"] == 2 and st["active"] == 0 and st["bytes_in_use"] == 0
    srv.cancel(b)
    assert srv.info(b)["state_name"] == "cancelled"
    with pytest.raises(N.LesgpuError):
        srv.cancel(b)
    with pytest.raises(N.LesgpuError):
        srv.result(a)                      # not finished
    st = srv.stats()
    assert st["queued"] == 1 and st["cancelled"] == 1 and st["latency_p50_s"] == -1.0
    with pytest.raises(N.LesgpuError):
        srv.submit(preset("c1"), 0)        # no steps
    srv.close()


def test_poisson_requests_match_the_serving_workload(S):
    r = S.poisson_requests(1000, rate=20.0, seed=3)
    t = np.array([q.t_arrival for q in r])
    assert np.all(np.diff(t) > 0)
    assert abs(1000 / t[-1] - 20.0) < 2.0
    grids = {(q.cfg.nx, q.cfg.ny, q.cfg.nz) for q in r}
    assert grids == {(64, 32, 32), (128, 64, 64), (192, 96, 96), (256, 128, 128)}
    ns = np.array([q.nsteps for q in r])
    assert ns.min() >= 500 and ns.max() <= 2000
    assert all(0.08 <= q.cfg.cs_unburned <= 0.22 for q in r)
    r2 = S.poisson_requests(1000, rate=20.0, seed=3)
    assert [q.cfg.as_dict() for q in r] == [q.cfg.as_dict() for q in r2]
