"""Multi-GPU plumbing of bench.py on CPU: two gloo ranks.

The covariance path does not shard (one dense Schur inverse per scene), so N
GPUs run N independent replicas; the only cross-rank steps are the barrier and
the max-over-ranks timing that turns per-rank times into one whole-job figure.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import sys
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        mine = 1.0 + rank  # rank 1 is the slow one
        t = bench.max_over_ranks(mine, "cpu")
        dist.barrier()
        out[rank] = (t, bench.replica_throughput(world, 10, t))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as man:
        out = man.dict()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    assert res[0] == res[1] == (2.0, 10.0)  # both ranks see the slowest time; 2 x 10 steps / 2 s


def test_single_process_is_identity():
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    assert bench.max_over_ranks(3.5, "cpu") == 3.5
    assert bench.replica_throughput(1, 7, 3.5) == pytest.approx(2.0)
