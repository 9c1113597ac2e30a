"""x-slab domain decomposition on the GPU (nuosc_b200.slabs).

All slabs of a solve live in this process on one GPU and swap their halo
planes with device copies before every RK stage (nuosc_halo_exchange_local),
the single-GPU stand-in for the NCCL exchange between processes (whose host
logic tests/test_slabs_cpu.py runs over gloo).  The decomposed solve equals
the undecomposed one bit for bit -- the stage kernels read the neighbours'
planes from the halo buffer instead of wrapping inside the register -- for 1,
2 and 3 slabs, FP64 and FP32, 6th- and 4th-difference KO, with the vacuum
term and with the tail kernel (642 velocities).
"""
import numpy as np
import pytest

import pyoracle as po

pytestmark = pytest.mark.gpu


def _whole(nb, n, nn, gx, precision, mu=1.3, pmo=0.3):
    x0, x1 = po.box(n, 0.1)
    s = nb.NuOsc(1, 1, nn, 0, gx, gx, x0, x1, x0, x1, 0.1, 0.1, 0.4, 0.1, precision=precision)
    s.set_mu(mu)
    s.set_pmo(pmo)
    return s


def _slabs(px, n, nn, gx, precision, mu=1.3, pmo=0.3):
    from nuosc_b200 import slabs
    x0, x1 = po.box(n, 0.1)
    s = slabs.LocalSlabs(px, nn, gx, x0, x1, x0, x1, 0.1, 0.1, 0.4, 0.1, precision=precision)
    s.set_mu(mu)
    s.set_pmo(pmo)
    return s


INIT = dict(alpha=1.2, eps0=1e-3, sigma=1.0, lnue=0.6, lnueb=0.4)


@pytest.mark.parametrize("px,nn,gx,precision", [(1, 4, 3, 0), (2, 8, 3, 0), (3, 4, 3, 0), (2, 4, 2, 0),
                                                 (3, 8, 3, 1), (2, 4, 3, 1)])
def test_slabs_equal_the_whole_solve(gpu, px, nn, gx, precision):
    import nuosc_b200 as nb
    n = 32
    w = _whole(nb, n, nn, gx, precision)
    w.fillInitValue(1, INIT["alpha"], INIT["eps0"], INIT["sigma"], INIT["lnue"], INIT["lnueb"], seed=41)
    w.step_rk4(8)
    ref = w.get_state()
    dref = w.analysis()
    n0 = np.array(w.n_nue0)
    w.close()
    s = _slabs(px, n, nn, gx, precision)
    s.fillInitValue(1, INIT["alpha"], INIT["eps0"], INIT["sigma"], INIT["lnue"], INIT["lnueb"], seed=41)
    s.step_rk4(8)
    got = s.get_state()
    assert got.shape == ref.shape
    assert np.array_equal(got.view(np.uint64), ref.view(np.uint64))
    d = s.analysis()
    for k in ("phy_time", "surv", "survb", "aM0", "Lex"):
        np.testing.assert_allclose(d[k], dref[k], rtol=1e-12, atol=1e-15)
    assert d["maxdP"] == dref["maxdP"]
    for sl in s.slabs:  # every slab holds the whole solve's initial number densities
        np.testing.assert_allclose(np.array(sl.n_nue0), n0, rtol=1e-12)
    s.close()


def test_single_slab_step_rk4_is_the_periodic_solve(gpu):
    """A solve of one slab (px = 1) steps with nuosc_step_rk4, its halo filled
    from its own boundary planes: bit-identical to the ordinary handle."""
    import nuosc_b200 as nb
    x0, x1 = po.box(32, 0.1)
    a = _whole(nb, 32, 4, 3, 0)
    b = nb.NuOsc(1, 1, 4, 0, 3, 3, x0, x1, x0, x1, 0.1, 0.1, 0.4, 0.1, slab_rank=0)
    b.set_mu(1.3)
    b.set_pmo(0.3)
    for s in (a, b):
        s.fillInitValue(1, INIT["alpha"], INIT["eps0"], INIT["sigma"], INIT["lnue"], INIT["lnueb"], seed=3)
        s.step_rk4(5)
    assert np.array_equal(a.get_state().view(np.uint64), b.get_state().view(np.uint64))
    a.close()
    b.close()


def test_slab_refusals(gpu):
    import nuosc_b200 as nb
    s = _slabs(2, 32, 2, 3, 0)
    with pytest.raises(nb.NuoscError) as e:
        s.slabs[0].step_rk4(1)  # two slabs: the caller drives stages and exchanges
    assert e.value.code == nb._lib.ERR_UNSUPPORTED
    with pytest.raises(nb.NuoscError):
        nb.Batch([s.slabs[0]])
    s.close()
    x0, x1 = po.box(32, 0.1)
    with pytest.raises(nb.NuoscError):  # slabs of 2 planes are thinner than the ghost width
        nb.NuOsc(16, 1, 2, 0, 3, 3, x0, x1, x0, x1, 0.1, 0.1, 0.4, 0.1, slab_rank=0)
