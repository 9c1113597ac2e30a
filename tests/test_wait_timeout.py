"""Failure detection on the GPU without a fault.

The stage kernels bound every mbarrier wait; when a wait runs out they
record the timeout in a status word, stop and return, and the host call
reports NUOSC_ERR_TIMEOUT.  nuosc_selftest_wait_timeout runs that wait on a
barrier that nothing completes: the test checks that it gives up, that the
timeout is reported, and that the device then still computes a solve that
agrees with the oracle.  nuosc_selftest_overdeclare_tx drives the TMA stage
kernels' own path -- a march whose box never completes (its byte count
over-declared; every real copy lands), the drain of the copies in flight,
the early return -- solo and inside a batch.
"""
import ctypes
import time

import pytest

import pyoracle as po


@pytest.mark.gpu
def test_bounded_wait_expires_and_is_reported(gpu):
    import nuosc_b200 as nb
    from nuosc_b200 import _lib
    ms = ctypes.c_double(-1.0)
    rc = nb.lib().nuosc_selftest_wait_timeout(0, 1 << 12, ctypes.byref(ms))
    assert rc == _lib.ERR_TIMEOUT
    assert b"expired" in nb.lib().nuosc_last_error()
    assert 0.0 < ms.value < 10000.0
    assert nb.lib().nuosc_selftest_wait_timeout(0, 0, None) == _lib.ERR_INVALID

    # the context is intact: a small solve afterwards matches the oracle
    x0, x1 = po.box(32, 0.1)
    s = nb.NuOsc(1, 1, 2, 0, 3, 3, x0, x1, x0, x1, 0.1, 0.1, 0.4, 0.1)
    s.set_mu(1.0)
    s.set_pmo(0.0)
    s.fillInitValue(1, 0.9, 1e-6, 1.0, 0.6, 0.5, seed=5)
    s.step_rk4(3)
    s.synchronize()
    st = s.get_state()
    s.close()
    o = po.Oracle(nn=2, x0=x0, x1=x1, z0=x0, z1=x1, dx=0.1, dz=0.1, cfl=0.4, ko=0.1, ko_order=6)
    o.fill_init(ipt=1, alpha=0.9, eps0=1e-6, lnue=0.6, lnueb=0.5, seed=5)
    o.step(3)
    ref = o.get_state(0)
    assert max(po.relerr(st[f], ref[f]) for f in range(8)) < 1e-12


def _small_solve(nb, x0, x1, seed=5):
    s = nb.NuOsc(1, 1, 2, 0, 3, 3, x0, x1, x0, x1, 0.1, 0.1, 0.4, 0.1)
    s.set_mu(1.0)
    s.set_pmo(0.0)
    s.set_kernel(nb.KERNEL_XTMA)
    s.fillInitValue(1, 0.9, 1e-6, 1.0, 0.6, 0.5, seed=seed)
    return s


@pytest.mark.gpu
@pytest.mark.parametrize("batched", [False, True])
def test_stage_kernel_timeout_path(gpu, batched):
    """One RK4 step with one box of the first tile over-declared in every TMA
    stage launch: each launch's bounded waits run out, the tile drains its
    copies and returns, the synchronize call reports NUOSC_ERR_TIMEOUT (once),
    and a fresh solve on the same handle then matches the oracle."""
    import nuosc_b200 as nb
    from nuosc_b200 import _lib
    x0, x1 = po.box(32, 0.1)
    s = _small_solve(nb, x0, x1)
    _lib.check(nb.lib().nuosc_selftest_overdeclare_tx(s.handle, 16))
    assert nb.lib().nuosc_selftest_overdeclare_tx(s.handle, 8) == _lib.ERR_INVALID
    t0 = time.time()
    if batched:
        b = nb.Batch([s])
        b.step_rk4(1)
        with pytest.raises(nb.NuoscError) as e:
            b.synchronize()
        b.close()
    else:
        s.step_rk4(1)
        with pytest.raises(nb.NuoscError) as e:
            s.synchronize()
    assert e.value.code == _lib.ERR_TIMEOUT
    assert time.time() - t0 < 120.0
    s.synchronize()  # reported once; the status word is clear again

    _lib.check(nb.lib().nuosc_selftest_overdeclare_tx(s.handle, 0))
    s.fillInitValue(1, 0.9, 1e-6, 1.0, 0.6, 0.5, seed=5)
    s.step_rk4(3)
    s.synchronize()
    st = s.get_state()
    s.close()
    o = po.Oracle(nn=2, x0=x0, x1=x1, z0=x0, z1=x1, dx=0.1, dz=0.1, cfl=0.4, ko=0.1, ko_order=6)
    o.fill_init(ipt=1, alpha=0.9, eps0=1e-6, lnue=0.6, lnueb=0.5, seed=5)
    o.step(3)
    ref = o.get_state(0)
    assert max(po.relerr(st[f], ref[f]) for f in range(8)) < 1e-12
