"""nuosc_b200 -- B200-native RK4 time step of nuosc's 2D-space x velocity-sphere
neutrino flavour kinetic equations.

`NuOsc` mirrors the reference's C++ class NuOsc (nuosc_class.h:99-191): same
constructor arguments, the same method names (set_mu, set_pmo, set_renorm,
fillInitValue, calRHS, vectorize, step_rk4, updatePeriodicBoundary, analysis,
addSnapShotAtV, addSnapShotAtXV, checkSnapShot) and the same meaning.  All of
them call the C ABI of include/nuosc_b200.h; the state lives in HBM.

    from nuosc_b200 import NuOsc
    s = NuOsc(1, 1, 4, 0, 3, 3, -3.2, 3.2, -3.2, 3.2, 0.1, 0.1, 0.4, 0.1)
    s.set_mu(1.0); s.set_pmo(0.0)
    s.fillInitValue(1, 0.9, 1e-6, 1.0, 0.6, 0.5, 0, 0, seed=7)
    for t in range(100):
        s.step_rk4()
    print(s.analysis())
"""
import ctypes as C
import math
import os

import numpy as np

from . import _lib
from ._lib import (FP32, FP64, KERNEL_AUTO, KERNEL_DIRECT, KERNEL_XMARCH, KERNEL_XTMA, LAYOUT_COMPACT,
                   LAYOUT_GHOSTED, REG_COR, REG_PRE, REG_RHS, REG_STAT, FIELDS, NuoscError, check, lib)

def release_cached_memory(device=0):
    """Return the device memory that destroyed handles left in the pool."""
    check(lib().nuosc_release_cached_memory(int(device)))


__all__ = ["NuOsc", "Batch", "release_cached_memory", "NuoscError", "FP32", "FP64", "REG_STAT", "REG_RHS", "REG_PRE", "REG_COR",
           "KERNEL_AUTO", "KERNEL_DIRECT", "KERNEL_XMARCH", "KERNEL_XTMA", "FIELDS", "lib"]

lib()  # fail at import time if the CUDA library is missing


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(seq):
    arr = (C.c_int * len(seq))(*[int(x) for x in seq])
    return arr


class Grid:
    """Geometry view (the reference's CartGrid members used by callers)."""

    def __init__(self, g, vx, vy, vz, vw):
        self.nx, self.nz, self.nv = g.nx, g.nz, g.nv
        self.nv_stride = g.nv_stride
        self.gx, self.gz = g.gx, g.gz
        self.x0, self.x1, self.z0, self.z1 = g.x0, g.x1, g.z0, g.z1
        self.dx, self.dz = g.dx, g.dz
        self.vx, self.vy, self.vz, self.vw = vx, vy, vz, vw
        self.X = g.x0 + (np.arange(g.nx) + 0.5) * g.dx  # CartGrid.cpp:199
        self.Z = g.z0 + (np.arange(g.nz) + 0.5) * g.dz  # CartGrid.cpp:200
        self.lpts = (g.nx + 2 * g.gx) * (g.nz + 2 * g.gz) * g.nv  # CartGrid.cpp:208

    def get_lpts(self):
        return self.lpts

    def idx(self, i, j, v):
        """Ghosted linear index of the reference (CartGrid.h:91)."""
        return ((i + self.gx) * (self.nz + 2 * self.gz) + j + self.gz) * self.nv + v


class NuOsc:
    """Drop-in for the reference's NuOsc on one B200 (nuosc_class.h:99-191).

    Constructor arguments are those of NuOsc::NuOsc (nuosc_class.cpp:454):
    px, pz (must be 1), nv (icosahedron subdivision count), nphi (unused),
    gx, gz (3: 6th-difference KO; 2: 4th-difference KO), the box x0, x1, z0,
    z1, spacings dx, dz, CFL and ko.  Extra keywords: precision (FP64 or
    FP32), device, and slab_rank: with px > 1 (pz = 1) the handle is x-slab
    `slab_rank` of the decomposed solve (nuosc_create_slab; see
    nuosc_b200.slabs), as the reference's constructor takes its rank from MPI.
    """

    def __init__(self, px, pz, nv, nphi, gx, gz, x0, x1, z0, z1, dx, dz, CFL, ko, precision=FP64, device=0,
                 slab_rank=None):
        p = _lib.Params(px=px, pz=pz, nv=nv, nphi=nphi, gx=gx, gz=gz, x0=x0, x1=x1, z0=z0, z1=z1, dx=dx, dz=dz,
                        cfl=CFL, ko=ko, precision=precision, device=device)
        h = C.c_void_p()
        if slab_rank is None:
            check(lib().nuosc_create(C.byref(p), C.byref(h)))
        else:
            check(lib().nuosc_create_slab(C.byref(p), int(slab_rank), C.byref(h)))
        self._h = h
        self.CFL, self.ko, self.precision = CFL, ko, precision
        self.mu, self.pmo, self.renorm = 1.0, 0.1, False  # NuOsc defaults (nuosc_class.h:124-126)
        g = self._geometry()
        nv_ = g.nv
        vx, vy, vz, vw = (np.zeros(nv_) for _ in range(4))
        check(lib().nuosc_get_velocities(h, _dp(vx), _dp(vy), _dp(vz), _dp(vw)))
        self.grid = Grid(g, vx, vy, vz, vw)
        self.dt, self.dx, self.dz, self.ds_L = g.dt, g.dx, g.dz, g.ds_L

    # ------------------------------------------------------------ lifetime
    def close(self):
        if getattr(self, "_h", None):
            check(lib().nuosc_destroy(self._h))  # refused while the handle is in a live Batch
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    # ------------------------------------------------------------ settings
    def set_mu(self, mu):
        self.mu = mu
        check(lib().nuosc_set_mu(self._h, mu))

    def set_pmo(self, pmo):
        self.pmo = pmo
        check(lib().nuosc_set_pmo(self._h, pmo))

    def set_renorm(self, renorm):
        self.renorm = bool(renorm)
        check(lib().nuosc_set_renorm(self._h, int(bool(renorm))))

    def set_kernel(self, kind):
        check(lib().nuosc_set_kernel(self._h, kind))

    def set_tile(self, tz, lx):
        check(lib().nuosc_set_tile(self._h, int(tz), int(lx)))

    def get_tile(self):
        tz, lx = C.c_int(), C.c_int()
        check(lib().nuosc_get_tile(self._h, C.byref(tz), C.byref(lx)))
        return tz.value, lx.value

    def set_moment_sum(self, msum):
        """FP32 TMA kernel: 1 sums the velocity-moment partials in FP64, 0 in float."""
        check(lib().nuosc_set_moment_sum(self._h, int(msum)))

    def get_moment_sum(self):
        m = C.c_int()
        check(lib().nuosc_get_moment_sum(self._h, C.byref(m)))
        return m.value

    def moment_error(self):
        """Relative summation error of the fused cell moments of v_stat against an
        FP64 recomputation from the stored state."""
        e = C.c_double()
        check(lib().nuosc_moment_error(self._h, C.byref(e)))
        return e.value

    def _geometry(self):
        g = _lib.Geometry()
        check(lib().nuosc_get_geometry(self._h, C.byref(g)))
        return g

    @property
    def phy_time(self):
        return self._geometry().phy_time

    @phy_time.setter
    def phy_time(self, t):
        check(lib().nuosc_set_time(self._h, t))

    @property
    def n_nue0(self):
        return tuple(self._geometry().n_nue0)

    @property
    def device_bytes(self):
        return self._geometry().device_bytes

    def get_lpts(self):
        return self.grid.lpts

    def get_nv(self):
        return self.grid.nv

    @property
    def G0(self):
        a, b = np.zeros(self.grid.nv), np.zeros(self.grid.nv)
        check(lib().nuosc_get_spectra(self._h, _dp(a), _dp(b)))
        return a

    @property
    def G0b(self):
        a, b = np.zeros(self.grid.nv), np.zeros(self.grid.nv)
        check(lib().nuosc_get_spectra(self._h, _dp(a), _dp(b)))
        return b

    def set_spectra(self, G0, G0b, n_nue0, n_nueb0):
        G0 = np.ascontiguousarray(G0, dtype=np.float64)
        G0b = np.ascontiguousarray(G0b, dtype=np.float64)
        check(lib().nuosc_set_spectra(self._h, _dp(G0), _dp(G0b), n_nue0, n_nueb0))

    # ------------------------------------------------------------ init / state
    def fillInitValue(self, ipt, alpha, eps0, sigma, lnue, lnueb, lnuex=0.0, lnuebx=0.0, seed=0):
        """nuosc_init.cpp:17-137: ipt 0..3 the generic branch (ipt=1 draws eps0*U(-1,1)
        per (x,z) from `seed`), ipt 4 the "NOC" Fourier-phase branch (phases
        from `seed`, every x), ipt 10/20/30 the advection tests (Advtest,
        Square, Triangle; eps0 and sigma only).  lnuex/lnuebx <= 0 (or inf)
        mean unbounded, the reference default."""
        lnuex = 0.0 if (lnuex is None or math.isinf(lnuex) or lnuex >= 1e300) else lnuex
        lnuebx = 0.0 if (lnuebx is None or math.isinf(lnuebx) or lnuebx >= 1e300) else lnuebx
        check(lib().nuosc_fill_init(self._h, int(ipt), alpha, eps0, sigma, lnue, lnueb, lnuex, lnuebx, int(seed)))

    def save_checkpoint(self, path):
        """Write the solve (state, spectra, time, moments) to `path`."""
        check(lib().nuosc_save_checkpoint(self._h, os.fsencode(path)))

    def load_checkpoint(self, path):
        """Restore a solve saved by save_checkpoint into this handle (same grid)."""
        check(lib().nuosc_load_checkpoint(self._h, os.fsencode(path)))

    def fillInitAdvtest(self, eps0, sigma):
        """NuOsc::fillInitAdvtest (nuosc_init.cpp:162-186): G0 = G0b = 1, ee a z profile."""
        self.fillInitValue(10, 0.0, eps0, sigma, 1.0, 1.0)

    def fillInitSquare(self, eps0, sigma):
        """NuOsc::fillInitSquare (nuosc_init.cpp:188-211)."""
        self.fillInitValue(20, 0.0, eps0, sigma, 1.0, 1.0)

    def fillInitTriangle(self, eps0, sigma):
        """NuOsc::fillInitTriangle (nuosc_init.cpp:213-236)."""
        self.fillInitValue(30, 0.0, eps0, sigma, 1.0, 1.0)

    def get_field(self, field, reg=REG_STAT, layout=LAYOUT_COMPACT):
        g = self.grid
        if layout == LAYOUT_COMPACT:
            out = np.zeros((g.nx, g.nz, g.nv))
        else:
            out = np.zeros(g.lpts)
        check(lib().nuosc_get_state(self._h, reg, field, _dp(out), layout))
        return out

    def get_state(self, reg=REG_STAT):
        """All 8 fields of a register as a (8, nx, nz, nv) float64 array."""
        return np.stack([self.get_field(f, reg) for f in range(8)])

    def set_field(self, field, arr, reg=REG_STAT, layout=LAYOUT_COMPACT):
        arr = np.ascontiguousarray(arr, dtype=np.float64)
        check(lib().nuosc_set_state(self._h, reg, field, _dp(arr), layout))

    def set_state(self, arr, reg=REG_STAT):
        for f in range(8):
            self.set_field(f, arr[f], reg)

    # ------------------------------------------------------------ hot path
    def updatePeriodicBoundary(self, reg=REG_STAT):
        check(lib().nuosc_update_periodic_boundary(self._h, reg))

    def calRHS(self, out=REG_RHS, inp=REG_STAT):
        check(lib().nuosc_calrhs(self._h, out, inp))

    def vectorize(self, dst, src1, a, src2, src3=None):
        if src3 is None:
            check(lib().nuosc_vectorize(self._h, dst, src1, a, src2))
        else:
            check(lib().nuosc_vectorize2(self._h, dst, src1, a, src2, src3))

    def step_rk4(self, nsteps=1):
        check(lib().nuosc_step_rk4(self._h, int(nsteps)))

    def synchronize(self):
        check(lib().nuosc_synchronize(self._h))

    @property
    def kernel_launches(self):
        return lib().nuosc_kernel_launches(self._h)

    @property
    def step_count(self):
        """RK4 steps since the initial data."""
        return lib().nuosc_step_count(self._h)

    def set_profiling(self, on=True):
        check(lib().nuosc_set_profiling(self._h, int(bool(on))))

    def get_profile(self):
        """{kind: (total_ms, launches)} since the last call (CUDA events on the handle's stream)."""
        n = len(_lib.PROF_KINDS)
        ms = np.zeros(n)
        cnt = (C.c_longlong * n)()
        check(lib().nuosc_get_profile(self._h, _dp(ms), cnt, n))
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(_lib.PROF_KINDS)}

    # ------------------------------------------------------------ analysis / output
    def analysis(self):
        d = _lib.Diag()
        check(lib().nuosc_analysis(self._h, C.byref(d)))
        return d.as_dict()

    def open_analysis_file(self, path="analysis.dat"):
        check(lib().nuosc_open_analysis_file(self._h, path.encode()))

    def addSnapShotAtV(self, var, fntpl, dumpstep, vidx):
        """var: field ids or names (FIELDS)."""
        f = [FIELDS.index(v) if isinstance(v, str) else int(v) for v in var]
        check(lib().nuosc_add_snapshot_at_v(self._h, _ip(f), len(f), fntpl.encode(), dumpstep, _ip(vidx),
                                            len(vidx)))

    def addSnapShotAtXV(self, var, fntpl, dumpstep, xidx, vidx):
        f = [FIELDS.index(v) if isinstance(v, str) else int(v) for v in var]
        check(lib().nuosc_add_snapshot_at_xv(self._h, _ip(f), len(f), fntpl.encode(), dumpstep, _ip(xidx),
                                             len(xidx), _ip(vidx), len(vidx)))

    def checkSnapShot(self, t=0):
        check(lib().nuosc_check_snapshot(self._h, int(t)))

    def gather(self, field, xidx, vidx):
        f = FIELDS.index(field) if isinstance(field, str) else int(field)
        out = np.zeros((len(xidx), self.grid.nz, len(vidx)))
        check(lib().nuosc_gather(self._h, f, _ip(xidx), len(xidx), _ip(vidx), len(vidx), _dp(out)))
        return out


class _PinnedRecords:
    """Page-locked nuosc_batch_record buffer (nuosc_host_alloc)."""

    def __init__(self, n):
        self.n = n
        self.used = 0
        self.ptr = lib().nuosc_host_alloc(n * C.sizeof(_lib.BatchRecord))
        if not self.ptr:
            raise MemoryError("nuosc_host_alloc failed")

    def at(self, k):
        return _lib.BatchRecord.from_address(self.ptr + k * C.sizeof(_lib.BatchRecord))

    def free(self):
        if self.ptr:
            lib().nuosc_host_free(self.ptr)
            self.ptr = None

    def __del__(self):
        self.free()


# Record buffers of closed batches, kept for the next batch: freeing page-locked
# memory (cudaFreeHost) waits for the whole device and measured up to 0.9 s
# per call in a serving loop, on the path between two quanta.
_REC_POOL = []
_REC_MIN = 1024  # records per buffer at least (about 0.2 MB)
_REC_POOL_MAX = 8


def _take_records(n):
    """A pooled record buffer of at least n records, or a new one."""
    fit = [b for b in _REC_POOL if b.n >= n]
    if fit:
        b = min(fit, key=lambda b: b.n)
        _REC_POOL.remove(b)
        return b
    return _PinnedRecords(max(n, _REC_MIN))


def _give_records(buf):
    """Return a batch's record buffer to the pool (the smallest are freed
    beyond _REC_POOL_MAX buffers)."""
    buf.used = 0
    _REC_POOL.append(buf)
    if len(_REC_POOL) > _REC_POOL_MAX:
        _REC_POOL.sort(key=lambda b: b.n)
        _REC_POOL.pop(0).free()


class Batch:
    """Several NuOsc instances stepped together (nuosc_batch_* of the C ABI).

    Each RK stage of a batch step is one persistent kernel over the tiles of
    all members, and the step is one CUDA graph replay; every member's state
    after `step_rk4(n)` is bit-for-bit what `member.step_rk4(n)` gives alone.
    Members must share device, precision and ghost width and have nz % 8 == 0,
    nz >= 14.  The batch keeps its members alive; close() (or the context
    manager) releases the batch, after which members can be closed.
    """

    def __init__(self, members):
        self.members = list(members)
        hs = (C.c_void_p * len(self.members))(*[m.handle for m in self.members])
        b = C.c_void_p()
        self._rec = None
        check(lib().nuosc_batch_create(hs, len(self.members), C.byref(b)))
        self._b = b

    def close(self):
        if getattr(self, "_b", None):
            lib().nuosc_batch_destroy(self._b)
            self._b = None
        if getattr(self, "_rec", None) is not None:
            _give_records(self._rec)
            self._rec = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._b

    def step_rk4(self, nsteps=1):
        check(lib().nuosc_batch_step(self._b, int(nsteps)))

    def step_stream(self, nsteps, every):
        """nsteps steps; the analysis of each member is queued on the device
        whenever its step count reaches a multiple of `every`.  Returns a
        handle for collect(), valid after synchronize(); the record buffer is
        the batch's own and is reused by the next step_stream, so collect the
        records first."""
        nmax = max(1, len(self.members) * (int(nsteps) // max(1, int(every)) + 1))
        if self._rec is None or self._rec.n < nmax:
            if self._rec is not None:
                _give_records(self._rec)
            self._rec = _take_records(max(nmax, 2 * len(self.members)))
        buf = self._rec
        n = C.c_int()
        check(lib().nuosc_batch_step_stream(self._b, int(nsteps), int(every), buf.ptr, buf.n, C.byref(n)))
        buf.used = n.value
        return buf

    def collect(self, records):
        """[(member index, step, analysis dict or None if the state blew up)]
        of a step_stream() handle; call after synchronize()."""
        out = []
        for k in range(records.used):
            r = records.at(k)
            d = _lib.Diag()
            rc = lib().nuosc_batch_record_diag(self._b, C.byref(r), C.byref(d))
            if rc not in (_lib.OK, _lib.ERR_NUMERIC):
                check(rc)
            out.append((r.member, r.step, d.as_dict() if rc == _lib.OK else None))
        records.used = 0
        return out

    def synchronize(self):
        check(lib().nuosc_batch_synchronize(self._b))

    def set_halt(self, check_every):
        """Stop a member on the device once its analysis (every `check_every`
        of its steps, and at every streamed record) shows a non-finite value
        or max||P|-1| >= 10, the reference's stop test; 0 turns it off."""
        check(lib().nuosc_batch_set_halt(self._b, int(check_every)))

    def halted(self):
        """Per member (creation order): the step at which it stopped, 0 while it runs (synchronises)."""
        n = len(self.members)
        out = (C.c_int * n)()
        check(lib().nuosc_batch_halted(self._b, out, n))
        return [int(v) for v in out]

    def stream(self):
        return lib().nuosc_batch_stream(self._b)

    def info(self):
        i = _lib.BatchInfo()
        check(lib().nuosc_batch_get_info(self._b, C.byref(i)))
        return i.as_dict()
