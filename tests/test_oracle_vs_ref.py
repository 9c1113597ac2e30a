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


# The reference's advection unit test (Makefile:24-30, `make test2d_advec`,
# UNITTEST with --gz 2): x, z in [-0.5, 0.5), dx = dz = 0.02, nn = 2, KO4
# with ko 0.8, cfl 0.25, mu = pmo = 0 (pure advection and dissipation),
# eps0 1, sigma 0.2.
ADV_N, ADV_DX = 50, 0.02


def _adv_pair(ko_order=4, n=ADV_N, ko=0.8):
    x0, x1 = po.box(n, ADV_DX)
    kw = dict(nn=2, x0=x0, x1=x1, z0=x0, z1=x1, dx=ADV_DX, dz=ADV_DX, cfl=0.25, ko=ko, ko_order=ko_order, mu=0.0,
              pmo=0.0)
    return po.Oracle(**kw), po.RefSim(**kw)


def _integrals(state, vw):
    """I1, I2 of the advection test (nuosc_ana.cpp:58-61) with G0 = 1."""
    ee = state[0]
    nor = vw.sum() * ee.shape[0] * ee.shape[1]
    return (ee * vw).sum() / nor, (ee * ee * vw).sum() / nor


@pytest.mark.parametrize("ipt", [10, 20, 30])
def test_advection_initial_data(ipt):
    o, r = _adv_pair()
    for s in (o, r):
        s.fill_init(ipt=ipt, eps0=1.0, sigma=0.2)
    assert po.relerr(o.get_state(0), r.get_state(0)) < 1e-15
    np.testing.assert_array_equal(o.velocities()[4], np.ones(o.shape[2]))


@pytest.mark.parametrize("ko_order", [4, 6])
def test_advection_steps_and_integrals(ko_order):
    """fillInitAdvtest advanced 20 steps: the state matches the reference build,
    the oracle's I1/I2 equal the ones of the reference's state, and I1 (the
    particle number) is conserved to rounding -- periodic central differences
    and KO sum to zero over the grid.  I2 falls under the 4th-difference KO;
    under the 6th-difference KO it grows: the reference's KO6 coefficient
    -ko/(64 dx) (nuosc_class.cpp:114-117) times the 6th difference (-64 on
    the grid-scale mode) amplifies that mode at the rate ko/dx, while its KO4
    (-ko/(16 dx) times +16) damps it."""
    o, r = _adv_pair(ko_order)
    for s in (o, r):
        s.fill_init(ipt=10, eps0=1.0, sigma=0.2)
    i0 = o.adv_integrals()
    o.step(20)
    r.step(20)
    a, b = o.get_state(0), r.get_state(0)
    for f in range(8):
        assert po.relerr(a[f], b[f]) < 1e-13, f
    i1 = o.adv_integrals()
    # sums of 10^5 terms in different orders (sequential in C, pairwise in numpy)
    np.testing.assert_allclose(i1, _integrals(b, o.velocities()[3]), rtol=1e-11)
    assert abs(i1[0] - i0[0]) < 1e-11 * abs(i0[0])  # to the rounding of a 10^5-term sum
    if ko_order == 4:
        assert i1[1] < i0[1]
    else:
        assert i1[1] > i0[1]


def test_noc_initial_data_against_reference():
    """ipt = 4 ("NOC" branch): the oracle, given the phases the reference
    draws with rand() after srand(seed) (one OpenMP thread, so the draws are
    in loop order), reproduces the reference's x = 0 column (the only one the
    reference fills), spectra included."""
    import ctypes
    import math
    libc = ctypes.CDLL(None)
    gomp = ctypes.CDLL("libgomp.so.1")
    nthreads = gomp.omp_get_max_threads()
    o, r = _pair(60, 2, 6)
    amax = 60 // 2 // 10
    libc.srand(4242)
    phi = [2.0 * math.pi * libc.rand() / 2147483647 for _ in range(2 * amax + 1)]
    try:
        gomp.omp_set_num_threads(1)
        libc.srand(4242)
        r.fill_init(ipt=4, alpha=0.9, eps0=1e-6, sigma=1.0, lnue=0.6, lnueb=0.5)
    finally:
        gomp.omp_set_num_threads(nthreads)
    o.set_noc_phases(phi)
    o.fill_init(ipt=4, alpha=0.9, eps0=1e-6, sigma=1.0, lnue=0.6, lnueb=0.5)
    a, b = o.get_state(0), r.get_state(0)
    assert po.relerr(a[:, 0], b[:, 0]) < 1e-15
    assert np.abs(a[2, 0]).max() > 1e-9  # the perturbation is there
    np.testing.assert_allclose(o.velocities()[4], r.velocities()[4][:o.shape[2]], rtol=1e-15)
