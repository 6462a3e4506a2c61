"""bench.py's multi-GPU arithmetic on CPU ranks: two gloo processes, one replica each; the
job value uses the slowest rank's time (max over ranks) and counts every rank's cells."""
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import sys
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import bench
    r, local, w = bench._dist("gloo")
    bench._barrier(w)
    ms_max, value = bench.replica_throughput(1000, 20, 10.0 + 5.0 * r, w)
    q.put((r, w, ms_max, value))
    import torch.distributed as dist
    dist.barrier()
    dist.destroy_process_group()


def test_replicas_take_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, w, ms_max, value in out:
        assert w == 2 and ms_max == 15.0
        assert value == pytest.approx(2 * 1000 * 20 / 0.015)


def test_single_rank_is_its_own_max():
    import sys
    sys.path.insert(0, ROOT)
    import bench
    assert bench.replica_throughput(10, 4, 2.0, 1) == (2.0, 10 * 4 / 0.002)
