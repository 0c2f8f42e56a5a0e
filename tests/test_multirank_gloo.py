"""The multi-rank (replicas-only) host path of bench.py over gloo on CPU,
world size 2: disjoint seeds per rank, the max-over-ranks timing, the
whole-job value, and the reference arm leaving ranks > 0 without work."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime
    import sys

    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "md-force-routines_b200")]
    import torch.distributed as dist

    import bench

    w, r, local = bench.dist_setup("gloo")
    assert (w, r, local) == (world, rank, rank)
    ms = bench.max_over_ranks(10.0 + 5.0 * rank, w, "cpu")
    seeds = list(range(bench.rank_first_seed(r, 20), bench.rank_first_seed(r, 20) + 20))
    gathered = [None] * w
    dist.all_gather_object(gathered, seeds)
    out[rank] = (ms, gathered)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_ranks_gloo():
    import bench

    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_worker, args=(world, port, out), nprocs=world, join=True,
                           start_method="spawn")
        res = dict(out)
    for rank in range(world):
        ms, gathered = res[rank]
        assert ms == 15.0  # the slower rank's time on every rank
        assert not set(gathered[0]) & set(gathered[1])  # disjoint ensembles
        assert gathered[0][0] == 1 and gathered[1][0] == 21
    # weak scaling: twice the particles over the slowest rank's time
    assert bench.job_value(2e5, 100, 2, 15.0) == pytest.approx(2e5 * 100 * 2 / 0.015)
