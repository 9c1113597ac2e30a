"""The C oracle against the reference's NuOsc compiled from its own sources
(oracle/_ref, built here by `make -C oracle ref`).  Skipped where the
reference build is absent."""
import numpy as np
import pytest

import pyoracle as po

pytestmark = pytest.mark.skipif(not (po.ref_available(6) and po.ref_available(4)),
                                reason="reference build oracle/_ref not present")


def _pair(n, nn, ko_order, mu=1.0, pmo=0.0, dx=0.1, ko=0.1):
    x0, x1 = po.box(n, dx)
    kw = dict(nn=nn, x0=x0, x1=x1, z0=x0, z1=x1, dx=dx, dz=dx, cfl=0.4, ko=ko, ko_order=ko_order, mu=mu, pmo=pmo)
    return po.Oracle(**kw), po.RefSim(**kw)


@pytest.mark.parametrize("ko_order,pmo,mu", [(6, 0.0, 1.0), (4, 0.0, 1.0), (6, 0.5, 0.7), (4, 1.0, 1.9)])
def test_calrhs_random_state(ko_order, pmo, mu):
    o, r = _pair(10, 2, ko_order, mu=mu, pmo=pmo)
    rng = np.random.default_rng(3)
    s = rng.uniform(-1, 1, size=(8,) + o.shape)
    o.set_state(s, 0)
    r.set_state(s, 0)
    o.calrhs()
    r.calrhs()
    a, b = o.get_state(1), r.get_state(1)
    for f in range(8):
        assert po.relerr(a[f], b[f]) < 1e-14


@pytest.mark.parametrize("ko_order", [6, 4])
def test_steps_match(ko_order):
    o, r = _pair(12, 2, ko_order)
    for s in (o, r):
        s.fill_init(ipt=1, alpha=0.9, eps0=1e-6, lnue=0.6, lnueb=0.5, seed=11)
    o.step(25)
    r.step(25)
    a, b = o.get_state(0), r.get_state(0)
    for f in range(8):
        assert po.relerr(a[f], b[f]) < 1e-13
    np.testing.assert_allclose(o.analysis()[[2, 3, 6, 7]], r.analysis()[[2, 3, 6, 7]], rtol=1e-12)


@pytest.mark.parametrize("ipt", [0, 2, 3])
def test_other_initial_data(ipt):
    o, r = _pair(8, 2, 6)
    for s in (o, r):
        s.fill_init(ipt=ipt, alpha=1.1, eps0=1e-3, sigma=0.3, lnue=0.6, lnueb=0.45, seed=0)
    assert po.relerr(o.get_state(0), r.get_state(0)) < 1e-15
    np.testing.assert_allclose(o.info()["n_nue0"], r.info()["n_nue0"], rtol=1e-13)
