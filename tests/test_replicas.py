"""Multi-GPU host logic of bench.py on CPU: one process per rank over gloo
(world size 2), as torchrun would launch them.  The replicas share no data;
the only collectives are the barrier and the max-over-ranks of the timed
region, and the whole-job value is all ranks' cell-steps over the slowest
rank's time."""
import os
import socket
import sys

import pytest

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist
    w, r, local = bench.dist_setup(backend="gloo")
    assert (w, r, local) == (world, rank, rank)
    bench.barrier(w)
    t = bench.max_over_ranks(10.0 + 5.0 * rank, w)  # rank-local "timed region" in ms
    out.put((rank, t, bench.replica_value(1000, 4, t, w)))
    bench.barrier(w)
    dist.destroy_process_group()


def test_two_replicas_over_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(out.get(timeout=5) for _ in range(2))
    for rank, t, v in res:
        assert t == pytest.approx(15.0)  # every rank sees the slowest rank's time
        assert v == pytest.approx(2 * 1000 * 4 / 0.015)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        os.environ.pop(k, None)
    assert bench.dist_setup() == (1, 0, 0)
    assert bench.max_over_ranks(3.0, 1) == 3.0
    assert bench.replica_value(10, 2, 1000.0, 1) == pytest.approx(20.0)
