"""The N>1 benchmark path on CPU: two gloo ranks run the replica plumbing of
bench.py (rendezvous, barrier, max over ranks, whole-job rate)."""
import os
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import bench
    r, w, dist = bench.dist_init(world, backend="gloo")
    assert (r, w) == (rank, world)
    bench.barrier(dist)
    ms = 100.0 + 50.0 * rank          # per-rank device time of the timed region
    mx = bench.dist_max(dist, ms)
    out[rank] = (mx, bench.aggregate(w, 1000, mx))
    dist.destroy_process_group()


def test_two_replicas_report_max_over_ranks():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = 29500 + os.getpid() % 2000
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        assert all(p.exitcode == 0 for p in procs)
        assert out[0] == out[1]
        mx, rate = out[0]
        assert mx == 150.0
        assert rate == pytest.approx(2 * 1000 / 0.150)
