"""Host logic of the x-slab decomposition on CPU (gloo, world size 2 and 3).

Each rank runs one x-slab of a 24x24 cells x 42 velocities solve in the
oracle, whose x ghosts are filled before every calRHS by the product's halo
exchange (nuosc_b200.slabs.exchange) over gloo -- the same call that moves the
GPU slabs' pieces over NCCL.  The slabs' states, concatenated in x, equal the
undecomposed oracle solve bit for bit after 6 RK4 steps (vacuum term and
seeded per-cell perturbation on: the draws use the global x index).
"""
import os
import socket
import sys

import numpy as np
import pytest

from conftest import ROOT

N, NN, STEPS, SEED = 24, 2, 6, 99
PHYS = dict(alpha=1.2, eps0=1e-3, sigma=1.0, lnue=0.6, lnueb=0.4)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import datetime

    import torch
    import torch.distributed as dist
    import pyoracle as po
    from nuosc_b200 import slabs

    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    x0, x1 = po.box(N, 0.1)
    xoff, nxl = slabs.split(N, world, rank)
    lx0 = x0 + xoff * 0.1
    o = po.Oracle(nn=NN, x0=lx0, x1=lx0 + (nxl + 0.5) * 0.1, z0=x0, z1=x1, dx=0.1, dz=0.1, cfl=0.4, ko=0.1,
                  ko_order=6, mu=1.3, pmo=0.2)
    assert o.shape[0] == nxl
    o.set_xoff(xoff)
    o.fill_init(ipt=1, seed=SEED, **PHYS)
    g, nv = 3, o.shape[2]
    PL = (N + 2 * g) * nv  # one ghosted x plane
    left, right = (rank - 1) % world, (rank + 1) % world

    def fill(stage, reg):
        views = [o.field(reg, f) for f in range(8)]
        t = lambda a: torch.from_numpy(a)  # noqa: E731  (shares the oracle's memory)
        slabs.exchange([t(v[g * PL:2 * g * PL]) for v in views], [t(v[nxl * PL:(nxl + g) * PL]) for v in views],
                       [t(v[0:g * PL]) for v in views], [t(v[(nxl + g) * PL:(nxl + 2 * g) * PL]) for v in views],
                       left, right, rank)

    o.step_slab(STEPS, fill)
    out.put((rank, o.get_state(0)))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_slab_exchange_reproduces_single_solve(world):
    import torch.multiprocessing as mp
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(out.get(timeout=300) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs)
    got = np.concatenate([res[r] for r in range(world)], axis=1)
    x0, x1 = po.box(N, 0.1)
    o = po.Oracle(nn=NN, x0=x0, x1=x1, z0=x0, z1=x1, dx=0.1, dz=0.1, cfl=0.4, ko=0.1, ko_order=6, mu=1.3, pmo=0.2)
    o.fill_init(ipt=1, seed=SEED, **PHYS)
    o.step(STEPS)
    assert np.array_equal(got, o.get_state(0))


def test_split_covers_the_planes():
    sys.path.insert(0, ROOT)
    from nuosc_b200 import slabs
    for nx, px in ((1024, 8), (130, 3), (24, 5)):
        parts = [slabs.split(nx, px, r) for r in range(px)]
        assert parts[0][0] == 0 and sum(n for _, n in parts) == nx
        assert all(parts[r][0] + parts[r][1] == parts[r + 1][0] for r in range(px - 1))
        assert max(n for _, n in parts) - min(n for _, n in parts) <= 1


def _reduce_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import datetime

    import torch.distributed as dist
    from nuosc_b200 import slabs

    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    q = np.arange(12, dtype=np.float64) * (rank + 1) + 0.25 * rank
    q[0] = [3.0, 7.5, 1.0][rank]  # max||P|-1| of this slab
    out.put((rank, slabs._reduce_sums(q)))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_diagnostic_sums_reduce_over_slabs(world):
    """The slabs' raw analysis sums combine as the whole solve's: the maximum
    for max||P|-1| (entry 0), the sum for every other entry (the weighted
    sums and the non-finite count), on every rank alike."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_reduce_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(out.get(timeout=300) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs)
    want = sum(np.arange(12, dtype=np.float64) * (r + 1) + 0.25 * r for r in range(world))
    want[0] = max([3.0, 7.5, 1.0][:world])
    for r in range(world):
        assert np.array_equal(res[r], want)
