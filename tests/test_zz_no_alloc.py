"""nuosc_calrhs_noalloc -- the right-hand side for callers that cannot allocate.

A host framework that reserves the device's memory for its own allocator and
hands plugins only buffers it allocated cannot let this library call
cudaMalloc: the allocation fails when the pool holds the memory, or breaks the
framework's accounting.  nuosc_calrhs_noalloc takes every buffer from the caller and
keeps its only scratch (the per-cell velocity moments) in a fixed device
array.  Here the test plays such a caller: it owns the device buffers (made
through torch), calls the entry point through the C ABI twice in a row with
different states, and checks each result against the library's calRHS entry
point on the same state, with the calRHS tolerance used elsewhere in tests/.

The file is named to be collected last, so that a failure here leaves every
other test already run.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CALRHS_TOL = 1e-13


class RhsDesc(C.Structure):
    _fields_ = [("nx", C.c_int), ("nz", C.c_int), ("nv", C.c_int), ("nv_stride", C.c_int),
                ("precision", C.c_int), ("ko_order", C.c_int),
                ("dx", C.c_double), ("dz", C.c_double), ("ko", C.c_double), ("mu", C.c_double),
                ("pmo", C.c_double),
                ("vx", C.c_void_p), ("vy", C.c_void_p), ("vz", C.c_void_p), ("vw", C.c_void_p)]


def relerr(a, b):
    d = float(np.max(np.abs(a - b)))
    m = float(np.max(np.abs(b)))
    return d / m if m > 0 else d


@pytest.mark.parametrize("precision,ko_order", [(0, 6), (1, 4)])
def test_calrhs_noalloc_matches_calrhs(gpu, precision, ko_order):
    import torch
    import nuosc_b200 as nb

    lib = nb.lib()
    fn = lib.nuosc_calrhs_noalloc
    fn.argtypes = [C.POINTER(RhsDesc), C.c_void_p, C.c_void_p, C.c_void_p]
    fn.restype = C.c_int

    n, nn, dx = 24, 4, 0.1
    L = n * dx / 2
    ghost = 3 if ko_order == 6 else 2
    s = nb.NuOsc(1, 1, nn, 0, ghost, ghost, -L, L, -L, L, dx, dx, 0.4, 0.1, precision=precision)
    s.set_mu(1.3)
    s.set_pmo(0.4)
    g = s.grid
    nvs = g.nv_stride
    dtype = torch.float64 if precision == nb.FP64 else torch.float32
    dev = torch.device("cuda", 0)

    def padded(a):
        out = np.zeros(nvs)
        out[:g.nv] = a
        return torch.tensor(out, dtype=torch.float64, device=dev)

    quad = [padded(a) for a in (g.vx, g.vy, g.vz, g.vw)]
    desc = RhsDesc(nx=g.nx, nz=g.nz, nv=g.nv, nv_stride=nvs, precision=precision, ko_order=ko_order,
                   dx=dx, dz=dx, ko=0.1, mu=1.3, pmo=0.4,
                   vx=quad[0].data_ptr(), vy=quad[1].data_ptr(), vz=quad[2].data_ptr(), vw=quad[3].data_ptr())
    stream = torch.cuda.current_stream(dev)

    for call, seed in enumerate((11, 12)):  # two calls in a row, different states
        state = np.random.default_rng(seed).uniform(-1.0, 1.0, size=(8, g.nx, g.nz, g.nv))
        # the library's calRHS entry point on its own registers
        s.set_state(state, nb.REG_STAT)
        s.calRHS(nb.REG_RHS, nb.REG_STAT)
        expect = s.get_state(nb.REG_RHS)
        # the caller-owned buffers for the allocation-free entry point
        host_in = np.zeros((8, g.nx, g.nz, nvs))
        host_in[..., :g.nv] = state
        d_in = torch.tensor(host_in, dtype=dtype, device=dev)
        d_out = torch.full((8, g.nx, g.nz, nvs), float("nan"), dtype=dtype, device=dev)
        rc = fn(C.byref(desc), d_in.data_ptr(), d_out.data_ptr(), stream.cuda_stream)
        assert rc == 0, lib.nuosc_last_error()
        torch.cuda.synchronize(dev)
        got = d_out.double().cpu().numpy()[..., :g.nv]
        for f in range(8):
            assert relerr(got[f], expect[f]) < CALRHS_TOL, (call, f)
    s.close()


def test_calrhs_noalloc_rejects_oversized_grid(gpu):
    import nuosc_b200 as nb
    lib = nb.lib()
    fn = lib.nuosc_calrhs_noalloc
    fn.argtypes = [C.POINTER(RhsDesc), C.c_void_p, C.c_void_p, C.c_void_p]
    fn.restype = C.c_int
    desc = RhsDesc(nx=512, nz=512, nv=42, nv_stride=42, precision=0, ko_order=6, dx=0.1, dz=0.1, ko=0.1,
                   mu=1.0, pmo=0.0, vx=1, vy=1, vz=1, vw=1)
    rc = fn(C.byref(desc), C.c_void_p(16), C.c_void_p(16), None)
    assert rc == nb._lib.ERR_INVALID
    assert b"65536" in lib.nuosc_last_error()


def test_calrhs_noalloc_rejects_bad_spacing(gpu):
    import nuosc_b200 as nb
    lib = nb.lib()
    fn = lib.nuosc_calrhs_noalloc
    fn.argtypes = [C.POINTER(RhsDesc), C.c_void_p, C.c_void_p, C.c_void_p]
    fn.restype = C.c_int
    for dx, mu in ((0.0, 1.0), (-0.1, 1.0), (float("nan"), 1.0), (0.1, float("inf"))):
        desc = RhsDesc(nx=16, nz=16, nv=42, nv_stride=42, precision=0, ko_order=6, dx=dx, dz=0.1, ko=0.1,
                       mu=mu, pmo=0.0, vx=1, vy=1, vz=1, vw=1)
        rc = fn(C.byref(desc), C.c_void_p(16), C.c_void_p(16), None)
        assert rc == nb._lib.ERR_INVALID, (dx, mu)
        assert b"spacing" in lib.nuosc_last_error()
