"""Host-side checks of the C ABI (no GPU): the library loads, exports every
entry point include/*.h declares, computes the velocity quadrature on the host
and rejects bad arguments with status codes instead of crashing."""
import ctypes as C
import glob
import os
import re

import numpy as np
import pytest

from conftest import ROOT, golden, has_gpu


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names.update(re.findall(r"\b(nuosc_\w+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    import nuosc_b200
    lib = nuosc_b200.lib()
    syms = declared_symbols()
    assert "nuosc_step_rk4" in syms and "nuosc_create" in syms
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


@pytest.mark.parametrize("nn", [1, 2, 4, 8])
def test_host_quadrature_bit_exact(nn):
    import nuosc_b200
    lib = nuosc_b200.lib()
    nv = 10 * nn * nn + 2
    arrs = [np.zeros(nv) for _ in range(4)]
    n = C.c_int()
    ptrs = [a.ctypes.data_as(C.POINTER(C.c_double)) for a in arrs]
    assert lib.nuosc_velocity_quadrature(nn, *ptrs, C.byref(n)) == 0
    assert n.value == nv
    g = golden("quadrature.npz")
    for name, a in zip(("vx", "vy", "vz", "vw"), arrs):
        assert np.array_equal(a, g[f"{name}_{nn}"])


def test_bad_arguments_return_codes():
    import nuosc_b200
    from nuosc_b200 import _lib
    lib = nuosc_b200.lib()
    assert lib.nuosc_velocity_quadrature(0, None, None, None, None, None) == _lib.ERR_INVALID
    assert lib.nuosc_step_rk4(None, 1) == _lib.ERR_INVALID
    assert lib.nuosc_analysis(None, None) == _lib.ERR_INVALID
    assert b"null" in lib.nuosc_last_error()
    b = C.c_void_p()
    assert lib.nuosc_batch_create(None, 0, C.byref(b)) == _lib.ERR_INVALID
    assert lib.nuosc_batch_create((C.c_void_p * 1)(None), 1, C.byref(b)) == _lib.ERR_INVALID
    assert not b.value
    assert lib.nuosc_batch_step(None, 1) == _lib.ERR_INVALID
    assert lib.nuosc_batch_synchronize(None) == _lib.ERR_INVALID
    assert lib.nuosc_batch_destroy(None) == _lib.OK
    base = dict(px=1, pz=1, nv=2, nphi=0, gx=3, gz=3, x0=-0.4, x1=0.4, z0=-0.4, z1=0.4, dx=0.1, dz=0.1, cfl=0.4,
                ko=0.1, precision=0, device=0)
    for bad, code in ((dict(px=2), _lib.ERR_UNSUPPORTED), (dict(gx=4, gz=4), _lib.ERR_INVALID),
                      (dict(gx=3, gz=2), _lib.ERR_INVALID), (dict(dx=0.0), _lib.ERR_INVALID),
                      (dict(precision=7), _lib.ERR_INVALID), (dict(nv=0), _lib.ERR_INVALID),
                      (dict(ko=float("nan")), _lib.ERR_INVALID), (dict(cfl=float("inf")), _lib.ERR_INVALID),
                      (dict(x1=float("inf")), _lib.ERR_INVALID), (dict(dz=-0.1), _lib.ERR_INVALID),
                      (dict(dx=1e-12), _lib.ERR_INVALID)):  # (0.8 / 1e-12 cells: more than an int holds)
        p = _lib.Params(**{**base, **bad})
        h = C.c_void_p()
        assert lib.nuosc_create(C.byref(p), C.byref(h)) == code
        assert not h.value
        if code == _lib.ERR_INVALID and "gx" not in bad and "precision" not in bad and "nv" not in bad:
            p = _lib.Params(**{**base, "px": 2, **bad})
            assert lib.nuosc_create_slab(C.byref(p), 0, C.byref(h)) == _lib.ERR_INVALID
            assert not h.value


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_create_without_device_fails_cleanly():
    import nuosc_b200
    with pytest.raises(nuosc_b200.NuoscError) as e:
        nuosc_b200.NuOsc(1, 1, 2, 0, 3, 3, -0.4, 0.4, -0.4, 0.4, 0.1, 0.1, 0.4, 0.1)
    assert e.value.code == 2
