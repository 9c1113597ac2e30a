"""Spatial domain decomposition of one solve into x-slabs.

Replaces the reference's CartGrid decomposition and halo exchange
(CartGrid.cpp:130-200, 330-440; nuosc_boundary.cpp:64-208) for a split in x
(the reference's `--np px 1`).  Slab r of px owns a contiguous range of x
planes (nx/px each, the first nx%px one more), all z and all velocities; x is
periodic across the slabs, z periodic inside each.  The stage kernels read
the R (= ghost width) planes beyond each side of a slab from a halo buffer,
so before every RK stage the slabs swap the boundary planes of that stage's
input register:

    recv_lo[f] <- left neighbour's send_hi[f]     (its last R planes of field f)
    recv_hi[f] <- right neighbour's send_lo[f]    (its first R planes)

for the 8 fields: 32 pieces per slab and stage, each R * nz * nv_stride
contiguous values (nuosc_halo_info).  `exchange` moves them with
torch.distributed point-to-point operations: NCCL between GPUs (one process
per GPU; the pieces are device memory of the slab, the receiving side is its
own halo buffer, so no kernel reads a peer's memory) or gloo on CPU tensors.
`SlabSolve` is one process's slab of a decomposed solve; `LocalSlabs` holds
all slabs of a solve in one process on one device and swaps their halos with
device copies (nuosc_halo_exchange_local).  Either way the decomposed solve
equals the undecomposed one bit for bit: every point sees the same
neighbour values and the same arithmetic.

Diagnostics are sums over cells: each slab's raw sums are reduced (maximum
for entry 0, sums for the rest) and turned into the analysis record with the
whole box's normalisation.
"""
import ctypes as C

import numpy as np

from . import FP64, NuOsc, _lib
from ._lib import check, lib

NPIECE = 8  # fields per side


def exchange(send_lo, send_hi, recv_lo, recv_hi, left, right, rank, group=None):
    """One halo exchange of a ring of x-slabs: recv_lo[f] <- left's send_hi[f],
    recv_hi[f] <- right's send_lo[f] for every field f.  The arguments are
    lists of equal-sized tensors (CUDA for NCCL, CPU for gloo); left, right and
    rank are ranks of `group`.  A slab that is its own neighbour (one slab)
    copies locally.  Sends to the right carry tag 2f, sends to the left 2f+1,
    so with two slabs (left == right) each piece still meets its place under
    gloo.  NCCL ignores tags and matches the operations between two ranks in
    the order they are issued; per field every rank issues send right,
    receive left, send left, receive right, so with two slabs rank a's sends
    to b (send_hi[f], then send_lo[f]) meet b's receives from a (recv_lo[f],
    then recv_hi[f]) in the same order."""
    import torch.distributed as dist
    if left == rank and right == rank:
        for f in range(len(send_lo)):
            recv_lo[f].copy_(send_hi[f])
            recv_hi[f].copy_(send_lo[f])
        return
    ops = []
    for f in range(len(send_lo)):
        ops.append(dist.P2POp(dist.isend, send_hi[f], right, group, 2 * f))
        ops.append(dist.P2POp(dist.irecv, recv_lo[f], left, group, 2 * f))
        ops.append(dist.P2POp(dist.isend, send_lo[f], left, group, 2 * f + 1))
        ops.append(dist.P2POp(dist.irecv, recv_hi[f], right, group, 2 * f + 1))
    for req in dist.batch_isend_irecv(ops):
        req.wait()


def split(nx, px, rank):
    """(first plane, planes) of slab `rank` of px over nx planes."""
    base, rem = divmod(nx, px)
    return rank * base + min(rank, rem), base + (1 if rank < rem else 0)


class _DeviceBytes:
    """A CUDA array interface over raw device bytes (a halo piece)."""

    def __init__(self, ptr, nbytes):
        self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def _halo_info(s, k):
    info = _lib.Halo()
    check(lib().nuosc_halo_info(s.handle, k, C.byref(info)))
    return info


def _reduce_sums(q, group=None):
    import torch
    import torch.distributed as dist
    t0 = torch.tensor(q[:1], dtype=torch.float64)
    t1 = torch.tensor(q[1:], dtype=torch.float64)
    if dist.get_backend(group) == "nccl":
        t0, t1 = t0.cuda(), t1.cuda()
    dist.all_reduce(t0, op=dist.ReduceOp.MAX, group=group)
    dist.all_reduce(t1, op=dist.ReduceOp.SUM, group=group)
    return np.concatenate([t0.cpu().numpy(), t1.cpu().numpy()])


def _diag(s, q):
    d = _lib.Diag()
    qa = np.ascontiguousarray(q, dtype=np.float64)
    check(lib().nuosc_diag_from_sums(s.handle, qa.ctypes.data_as(C.POINTER(C.c_double)), C.byref(d)))
    return d.as_dict()


def _sums(s):
    q = np.zeros(12)
    check(lib().nuosc_analysis_sums(s.handle, q.ctypes.data_as(C.POINTER(C.c_double))))
    return q


class SlabSolve:
    """This process's x-slab of a solve decomposed over the ranks of a
    torch.distributed group (one GPU per rank).  Same constructor arguments
    as NuOsc (nn = icosahedron subdivisions, ghost width gx = gz, the whole
    box and spacing); the slab is rank r of the group's size."""

    def __init__(self, nn, gx, x0, x1, z0, z1, dx, dz, CFL, ko, precision=FP64, device=0, group=None):
        import torch.distributed as dist
        self.group = group
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.slab = NuOsc(self.world, 1, nn, 0, gx, gx, x0, x1, z0, z1, dx, dz, CFL, ko, precision=precision,
                          device=device, slab_rank=self.rank)
        self._pieces = {}

    def close(self):
        self.slab.close()

    def set_mu(self, mu):
        self.slab.set_mu(mu)

    def set_pmo(self, pmo):
        self.slab.set_pmo(pmo)

    def fillInitValue(self, *args, **kw):
        """NuOsc.fillInitValue on the slab; n_nue0 becomes the whole solve's."""
        self.slab.fillInitValue(*args, **kw)
        n = np.array(self.slab.n_nue0, dtype=np.float64)
        if self.world > 1:
            import torch
            import torch.distributed as dist
            t = torch.tensor(n)
            if dist.get_backend(self.group) == "nccl":
                t = t.cuda()
            dist.all_reduce(t, group=self.group)
            n = t.cpu().numpy()
        check(lib().nuosc_set_n_nue0(self.slab.handle, float(n[0]), float(n[1])))

    def _tensors(self, k):
        if k not in self._pieces:
            import torch
            info = _halo_info(self.slab, k)
            mk = lambda p: torch.as_tensor(_DeviceBytes(p, info.bytes), device="cuda")  # noqa: E731
            self._pieces[k] = ([mk(p) for p in info.send_lo], [mk(p) for p in info.send_hi],
                               [mk(p) for p in info.recv_lo], [mk(p) for p in info.recv_hi], info.left, info.right)
        return self._pieces[k]

    def step_rk4(self, nsteps=1):
        """nsteps RK4 steps: per stage, the halo exchange of its input, then the stage."""
        import torch
        stream = torch.cuda.ExternalStream(lib().nuosc_stream(self.slab.handle))
        for _ in range(nsteps):
            for k in range(4):
                slo, shi, rlo, rhi, left, right = self._tensors(k)
                with torch.cuda.stream(stream):
                    exchange(slo, shi, rlo, rhi, left, right, self.rank, self.group)
                check(lib().nuosc_stage(self.slab.handle, k))

    def analysis(self):
        """The whole solve's analysis record (the slabs' sums reduced)."""
        q = _sums(self.slab)
        if self.world > 1:
            q = _reduce_sums(q, self.group)
        return _diag(self.slab, q)

    def get_state(self, reg=0):
        """This slab's planes of the state, (8, nx_slab, nz, nv)."""
        return self.slab.get_state(reg)


class LocalSlabs:
    """All px x-slabs of one solve in this process on one device, stepped
    together with their halos copied on the device
    (nuosc_halo_exchange_local).  Equal, bit for bit, to the undecomposed
    solve: the test of the decomposition on one GPU."""

    def __init__(self, px, nn, gx, x0, x1, z0, z1, dx, dz, CFL, ko, precision=FP64, device=0):
        self.slabs = [NuOsc(px, 1, nn, 0, gx, gx, x0, x1, z0, z1, dx, dz, CFL, ko, precision=precision,
                            device=device, slab_rank=r) for r in range(px)]
        self._arr = (C.c_void_p * px)(*[s.handle for s in self.slabs])

    def close(self):
        for s in self.slabs:
            s.close()

    def set_mu(self, mu):
        for s in self.slabs:
            s.set_mu(mu)

    def set_pmo(self, pmo):
        for s in self.slabs:
            s.set_pmo(pmo)

    def fillInitValue(self, *args, **kw):
        for s in self.slabs:
            s.fillInitValue(*args, **kw)
        n = np.sum([s.n_nue0 for s in self.slabs], axis=0)
        for s in self.slabs:
            check(lib().nuosc_set_n_nue0(s.handle, float(n[0]), float(n[1])))

    def step_rk4(self, nsteps=1):
        for _ in range(nsteps):
            for k in range(4):
                check(lib().nuosc_halo_exchange_local(self._arr, len(self.slabs), k))
                for s in self.slabs:
                    check(lib().nuosc_stage(s.handle, k))

    def analysis(self):
        qs = [_sums(s) for s in self.slabs]
        q = np.sum(qs, axis=0)
        q[0] = max(x[0] for x in qs)
        return _diag(self.slabs[0], q)

    def get_state(self, reg=0):
        """The whole state, slabs concatenated in x: (8, nx, nz, nv)."""
        return np.concatenate([s.get_state(reg) for s in self.slabs], axis=1)
