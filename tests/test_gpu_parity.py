"""Parity of the CUDA path (through the C ABI) with the reference.

Fixtures in tests/golden/ come from the reference's own build; the oracle
(oracle/nuosc_oracle.c, pinned against that build by test_oracle.py) checks
larger cases.  The FP64 bar is the norm-wise relative error
    max|gpu - ref| / max|ref|  per field
after the stated number of RK4 steps:
    FP64_TOL = 1e-12 (state), CALRHS_TOL = 1e-13 (one right-hand side).
Diagnostics are sums over 10^4..10^7 terms; their summation order differs
(tree reduction on the device, sequential or OpenMP on the host), which alone
moves the O(1) sums by up to ~1e-11 relative, so DIAG_RTOL = 1e-10 there.
"""
import os

import numpy as np
import pytest

import pyoracle as po
from conftest import golden

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
CALRHS_TOL = 1e-13
DIAG_RTOL = 1e-10
PHYS = dict(alpha=0.9, eps0=1e-6, sigma=1.0, lnue=0.6, lnueb=0.5)


@pytest.fixture(scope="module")
def nb(gpu):
    import nuosc_b200
    return nuosc_b200


def make(nb, params, ko_order, precision=0, kernel=None):
    x0, x1, dx, cfl, ko, mu, pmo, nn = [float(p) for p in params]
    g = 3 if ko_order == 6 else 2
    s = nb.NuOsc(1, 1, int(nn), 0, g, g, x0, x1, x0, x1, dx, dx, cfl, ko, precision=precision)
    s.set_mu(mu)
    s.set_pmo(pmo)
    if kernel is not None:
        s.set_kernel(kernel)
    return s


def box_params(n, nn, dx=0.1, cfl=0.4, ko=0.1, mu=1.0, pmo=0.0):
    x0, x1 = po.box(n, dx)
    return (x0, x1, dx, cfl, ko, mu, pmo, nn)


def diag_vec(d):
    return np.array([d[k] for k in po.DIAG_NAMES])


def assert_diag_close(a, ref):
    np.testing.assert_allclose(a[[0, 2, 3, 6, 7]], ref[[0, 2, 3, 6, 7]], rtol=DIAG_RTOL)
    np.testing.assert_allclose(a[[1, 4, 5]], ref[[1, 4, 5]], atol=1e-13, rtol=1e-4)
    # ELNe = |n0 (1 - surv) - n1 (1 - survb)| / (n0 + n1) with 1 - surv ~ 1e-12:
    # pure cancellation, set by the last bits of surv
    np.testing.assert_allclose(a[8], ref[8], atol=1e-11)


KERNELS = [1, 2, 3]  # direct, cp.async x-march, TMA x-march


def _kernel_ok(nb, s, kernel):
    if kernel == nb.KERNEL_DIRECT:
        s.set_kernel(kernel)
    if kernel in (nb.KERNEL_XMARCH, nb.KERNEL_XTMA):
        try:
            s.step_rk4(0)
            s.set_kernel(kernel)
            s.step_rk4(0)
        except nb.NuoscError as e:
            if e.code == 6:
                pytest.skip("x-march kernel not available for this geometry")
            raise


@pytest.mark.parametrize("ko_order", [6, 4])
def test_init_matches_reference(nb, ko_order):
    g = golden(f"run_ko{ko_order}.npz")
    s = make(nb, g["params"], ko_order)
    s.fillInitValue(1, seed=int(g["seed"]), **PHYS)
    st = s.get_state()
    assert po.relerr(st, g["state0"]) < 1e-15
    np.testing.assert_allclose(s.n_nue0, g["n_nue0"], rtol=1e-13)
    np.testing.assert_allclose(s.G0, g["G0"], rtol=1e-15)
    np.testing.assert_allclose(s.G0b, g["G0b"], rtol=1e-15)


@pytest.mark.parametrize("ko_order", [6, 4])
def test_calrhs_matches_reference(nb, ko_order):
    g = golden(f"calrhs_ko{ko_order}.npz")
    s = make(nb, g["params"], ko_order)
    s.set_state(g["inp"], nb.REG_STAT)
    s.updatePeriodicBoundary(nb.REG_STAT)
    s.calRHS(nb.REG_RHS, nb.REG_STAT)
    rhs = s.get_state(nb.REG_RHS)
    for f in range(8):
        assert po.relerr(rhs[f], g["rhs"][f]) < CALRHS_TOL, f


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("ko_order", [6, 4])
def test_ten_steps_match_reference(nb, ko_order, kernel):
    g = golden(f"run_ko{ko_order}.npz")
    s = make(nb, g["params"], ko_order)
    s.fillInitValue(1, seed=int(g["seed"]), **PHYS)
    _kernel_ok(nb, s, kernel)
    a0 = diag_vec(s.analysis())
    s.step_rk4(10)
    st = s.get_state()
    for f in range(8):
        assert po.relerr(st[f], g["state10"][f]) < FP64_TOL, f
    a1 = diag_vec(s.analysis())
    assert_diag_close(a0, g["ana0"])
    assert_diag_close(a1, g["ana10"])


@pytest.mark.parametrize("kernel", KERNELS)
def test_series_64x64x162_100_steps(nb, kernel):
    """64x64 cells x 162 velocities, dx 0.1, 100 steps, analysis every 10:
    diagnostics against the reference's series, state against the oracle."""
    g = golden("series_64x64x162.npz")
    p = box_params(64, 4)
    s = make(nb, p, 6)
    s.fillInitValue(1, seed=int(g["seed"]), **PHYS)
    _kernel_ok(nb, s, kernel)
    series = [diag_vec(s.analysis())]
    for _ in range(10):
        s.step_rk4(10)
        series.append(diag_vec(s.analysis()))
    series = np.array(series)
    ref = g["series"]
    np.testing.assert_allclose(series[:, [0, 2, 3, 6, 7]], ref[:, [0, 2, 3, 6, 7]], rtol=DIAG_RTOL)
    np.testing.assert_allclose(series[:, 1], ref[:, 1], rtol=1e-4, atol=1e-14)
    flat = s.get_state().reshape(8, -1)
    np.testing.assert_allclose(flat.sum(axis=1), g["fsum"], rtol=1e-12, atol=1e-12 * g["fmax"].max())
    o = po.Oracle(nn=4, x0=p[0], x1=p[1], z0=p[0], z1=p[1], dx=0.1, dz=0.1, cfl=0.4, ko=0.1, ko_order=6)
    o.fill_init(ipt=1, seed=int(g["seed"]), **PHYS)
    o.step(100)
    ref_state = o.get_state(0).reshape(8, -1)
    for f in range(8):
        assert po.relerr(flat[f], ref_state[f]) < FP64_TOL, f


@pytest.mark.slow
@pytest.mark.parametrize("kernel", KERNELS)
def test_128_cells_162_velocities_100_steps(nb, kernel):
    """The parity size of the production configuration (128^2 x 162)."""
    p = box_params(128, 4)
    s = make(nb, p, 6)
    s.fillInitValue(1, seed=77, **PHYS)
    _kernel_ok(nb, s, kernel)
    s.step_rk4(100)
    st = s.get_state()
    o = po.Oracle(nn=4, x0=p[0], x1=p[1], z0=p[0], z1=p[1], dx=0.1, dz=0.1, cfl=0.4, ko=0.1, ko_order=6)
    o.fill_init(ipt=1, seed=77, **PHYS)
    o.step(100)
    ref = o.get_state(0)
    for f in range(8):
        assert po.relerr(st[f], ref[f]) < FP64_TOL, f
    assert_diag_close(diag_vec(s.analysis()), o.analysis())


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("n,nn", [(8, 1), (12, 2), (20, 2), (24, 4)])
def test_odd_sizes_against_oracle(nb, n, nn, kernel):
    """Sizes that do not divide the tile shapes, nv with a partial velocity block."""
    p = box_params(n, nn, mu=1.3, pmo=0.2)
    s = make(nb, p, 6)
    s.fillInitValue(1, seed=3, alpha=1.2, eps0=1e-3, sigma=1.0, lnue=0.6, lnueb=0.4)
    _kernel_ok(nb, s, kernel)
    s.step_rk4(7)
    o = po.Oracle(nn=nn, x0=p[0], x1=p[1], z0=p[0], z1=p[1], dx=0.1, dz=0.1, cfl=0.4, ko=0.1, ko_order=6, mu=1.3,
                  pmo=0.2)
    o.fill_init(ipt=1, seed=3, alpha=1.2, eps0=1e-3, sigma=1.0, lnue=0.6, lnueb=0.4)
    o.step(7)
    a, b = s.get_state(), o.get_state(0)
    for f in range(8):
        assert po.relerr(a[f], b[f]) < FP64_TOL, f


@pytest.mark.parametrize("ko_order", [6, 4])
def test_xmarch_tiles_bit_identical(nb, ko_order):
    """Every x-march tile shape gives the same bits (moment partials are reduced
    per 32-velocity block in a fixed order, independent of the tile), and the
    result matches the oracle."""
    p = box_params(40, 4)
    ref_bits = None
    for tz, lx in ((16, 128), (8, 128), (16, 7), (8, 1), (16, 40), (8, 13)):
        s = make(nb, p, ko_order)
        s.fillInitValue(1, seed=5, alpha=1.2, eps0=1e-3, sigma=1.0, lnue=0.6, lnueb=0.4)
        s.set_kernel(nb.KERNEL_XMARCH)
        s.set_tile(tz, lx)
        s.step_rk4(6)
        st = s.get_state()
        if ref_bits is None:
            ref_bits = st
            o = po.Oracle(nn=4, x0=p[0], x1=p[1], z0=p[0], z1=p[1], dx=0.1, dz=0.1, cfl=0.4, ko=0.1,
                          ko_order=ko_order)
            o.fill_init(ipt=1, seed=5, alpha=1.2, eps0=1e-3, sigma=1.0, lnue=0.6, lnueb=0.4)
            o.step(6)
            ref = o.get_state(0)
            for f in range(8):
                assert po.relerr(st[f], ref[f]) < FP64_TOL, f
        else:
            assert np.array_equal(st, ref_bits), (tz, lx)
        s.close()


def test_state_roundtrip_layouts(nb):
    p = box_params(8, 2)
    for prec in (nb.FP64, nb.FP32):
        s = make(nb, p, 6, precision=prec)
        rng = np.random.default_rng(0)
        st = rng.standard_normal((8, 8, 8, 42))
        s.set_state(st, nb.REG_PRE)
        back = s.get_state(nb.REG_PRE)
        if prec == nb.FP64:
            assert np.array_equal(back, st)
        else:
            assert np.array_equal(back, st.astype(np.float32).astype(np.float64))
        gh = s.get_field(3, nb.REG_PRE, layout=1)
        gxz = gh.reshape(8 + 6, 8 + 6, 42)[3:-3, 3:-3]
        np.testing.assert_array_equal(gxz, back[3])
        gh2 = np.zeros_like(gh)
        gh2.reshape(14, 14, 42)[3:-3, 3:-3] = st[5]
        s.set_field(5, gh2, nb.REG_COR, layout=1)
        np.testing.assert_array_equal(s.get_field(5, nb.REG_COR), back[5])


def test_vectorize(nb):
    p = box_params(8, 2)
    s = make(nb, p, 6)
    rng = np.random.default_rng(1)
    a, b, c = (rng.standard_normal((8, 8, 8, 42)) for _ in range(3))
    s.set_state(a, 1)
    s.set_state(b, 2)
    s.set_state(c, 3)
    s.vectorize(0, 1, 0.25, 2)
    np.testing.assert_allclose(s.get_state(0), a + 0.25 * b, rtol=0, atol=1e-15)
    s.vectorize(0, 1, 0.5, 2, 3)
    np.testing.assert_allclose(s.get_state(0), a + 0.5 * (b + c), rtol=0, atol=1e-15)


def test_snapshot_files_match_reference(nb, tmp_path):
    g = golden("snapshot.npz")
    s = make(nb, box_params(8, 2), 6)
    s.fillInitValue(1, seed=5, **PHYS)
    assert po.relerr(s.get_state(), g["state0"]) < 1e-15
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        s.addSnapShotAtV([0, 2], "ee%06d.bin", 1, [0, 21, 41])
        s.addSnapShotAtXV([4, 6, 3], "xv%06d.bin", 1, [1, 4], [3, 7, 40])
        s.checkSnapShot(0)
    finally:
        os.chdir(cwd)
    for name in ("ee000000.bin", "ee000000.bin.meta", "xv000000.bin", "xv000000.bin.meta"):
        mine = (tmp_path / name).read_bytes()
        assert mine == g[name.replace(".", "_")].tobytes(), name
    # a file-name template is a format given the step alone
    for bad in ("ee%s.bin", "ee%d_%d.bin", "ee%ld.bin", "ee%*d.bin"):
        with pytest.raises(nb.NuoscError) as e:
            s.addSnapShotAtV([0], str(tmp_path / bad), 1, [0])
        assert e.value.code == nb._lib.ERR_INVALID


def test_gather_derived_fields(nb):
    p = box_params(8, 2)
    s = make(nb, p, 6)
    s.fillInitValue(1, seed=9, alpha=1.1, eps0=1e-2, sigma=1.0, lnue=0.6, lnueb=0.5)
    s.step_rk4(3)
    st = s.get_state()
    G0, G0b = s.G0, s.G0b
    P3 = (st[0] - st[1]) / G0
    P2b = 2 * st[7] / G0b
    xi, vi = [0, 5], [1, 17, 40]
    np.testing.assert_allclose(s.gather("P3", xi, vi), P3[xi][:, :, vi], rtol=1e-14, atol=1e-15)
    np.testing.assert_allclose(s.gather("P2b", xi, vi), P2b[xi][:, :, vi], rtol=1e-14, atol=1e-15)
    P = np.sqrt((2 * st[2] / G0) ** 2 + (2 * st[3] / G0) ** 2 + P3 ** 2)
    np.testing.assert_allclose(s.gather("dP", xi, vi), np.abs(1 - P)[xi][:, :, vi], atol=1e-15)


def test_analysis_file_format(nb, tmp_path):
    s = make(nb, box_params(8, 2), 6)
    s.fillInitValue(1, seed=1, **PHYS)
    path = str(tmp_path / "analysis.dat")
    s.open_analysis_file(path)
    s.analysis()
    s.step_rk4(2)
    d = s.analysis()
    lines = open(path).read().splitlines()
    assert lines[0].startswith("### [ phy_time")
    vals = [float(x) for x in lines[-1].split()]
    assert len(vals) == 9
    np.testing.assert_allclose(vals[1:], [d[k] for k in po.DIAG_NAMES[1:]], rtol=1e-12, atol=1e-25)


def test_error_paths(nb):
    s = make(nb, box_params(8, 2), 6)
    with pytest.raises(nb.NuoscError) as e:
        s.calRHS(nb.REG_STAT, nb.REG_STAT)
    assert e.value.code == 1
    with pytest.raises(nb.NuoscError):
        s.updatePeriodicBoundary(7)
    with pytest.raises(nb.NuoscError) as e:
        s.fillInitValue(5, **PHYS)
    assert e.value.code == 6
    # a non-finite state is reported by analysis() as a numeric error
    s.fillInitValue(1, seed=1, **PHYS)
    st = s.get_state()
    st[2, 3, 4, 5] = np.nan
    s.set_state(st)
    with pytest.raises(nb.NuoscError) as e:
        s.analysis()
    assert e.value.code == 4


def test_fp32_tracks_fp64(nb):
    """FP32 state (FP64 cell moments and diagnostics) stays close to FP64 on
    64x64 cells x 162 velocities over 100 steps."""
    p = box_params(64, 4)
    runs = {}
    for prec in (nb.FP64, nb.FP32):
        s = make(nb, p, 6, precision=prec)
        s.fillInitValue(1, seed=2024, **PHYS)
        series = [diag_vec(s.analysis())]
        for _ in range(10):
            s.step_rk4(10)
            series.append(diag_vec(s.analysis()))
        runs[prec] = np.array(series)
    d = np.abs(runs[nb.FP32] - runs[nb.FP64])
    assert d[:, 2].max() < 1e-6      # Pee
    assert d[:, 4].max() < 1e-6      # <|P|-1>
    assert d[:, 6].max() < 1e-6      # |M0|


FP32_TOL = 2e-5  # norm-wise, FP32 state after 10 steps against the FP64 oracle


@pytest.mark.parametrize("n,nn,pmo", [(32, 4, 0.0), (32, 4, 0.3), (16, 8, 0.0)])
def test_fp32_kernels_against_oracle(nb, n, nn, pmo):
    """FP32 state (two velocities per thread in the TMA kernel, one in the
    others), FP64 cell moments: every stage kernel stays within FP32 rounding of the
    FP64 oracle on 32x32 x 162 and on 16x16 x 642, where the TMA path hands
    the last velocity block, 640-641 and the zero padding 642-643, to the tail
    kernel."""
    p = box_params(n, nn, pmo=pmo)
    o = po.Oracle(nn=nn, x0=p[0], x1=p[1], z0=p[0], z1=p[1], dx=0.1, dz=0.1, cfl=0.4, ko=0.1, ko_order=6, pmo=pmo)
    o.fill_init(ipt=1, seed=8, alpha=1.2, eps0=1e-3, sigma=1.0, lnue=0.6, lnueb=0.4)
    o.step(10)
    ref = o.get_state(0)
    for kernel in KERNELS:
        s = make(nb, p, 6, precision=nb.FP32)
        s.fillInitValue(1, seed=8, alpha=1.2, eps0=1e-3, sigma=1.0, lnue=0.6, lnueb=0.4)
        s.set_kernel(kernel)
        s.step_rk4(10)
        st = s.get_state()
        for f in range(8):
            assert po.relerr(st[f], ref[f]) < FP32_TOL, (kernel, f)
        s.close()


def test_launch_count(nb):
    s = make(nb, box_params(16, 2), 6)
    s.fillInitValue(1, seed=1, **PHYS)
    n0 = s.kernel_launches
    s.step_rk4(3)
    assert s.kernel_launches - n0 >= 3 * 4


def _tma_solve(nb, p, ko_order, seed, steps, tile=None, **phys):
    """Runs `steps` RK4 steps on the TMA x-march kernel, which must accept the
    geometry (no silent fallback to another kernel)."""
    s = make(nb, p, ko_order, kernel=nb.KERNEL_XTMA)
    if tile is not None:
        s.set_tile(*tile)
    s.fillInitValue(1, seed=seed, **phys)
    s.step_rk4(steps)
    return s


def _oracle_solve(p, ko_order, seed, steps, ipt=1, **phys):
    x0, x1, dx, cfl, ko, mu, pmo, nn = p
    o = po.Oracle(nn=int(nn), x0=x0, x1=x1, z0=x0, z1=x1, dx=dx, dz=dx, cfl=cfl, ko=ko, ko_order=ko_order, mu=mu,
                  pmo=pmo)
    o.fill_init(ipt=ipt, seed=seed, **phys)
    if steps:
        o.step(steps)
    return o


HARD = dict(alpha=1.2, eps0=1e-3, sigma=1.0, lnue=0.6, lnueb=0.4)


@pytest.mark.parametrize("pmo", [0.0, 0.3])
def test_tma_fp64_642_velocities_against_oracle(nb, pmo):
    """The production kernel configuration on a small grid: FP64, 642
    velocities (nn = 8: 20 full 32-velocity blocks on the TMA kernel, 640-641
    on the tail kernel), 16-row tiles with the tile table's 128-plane x
    segments, 6th-difference KO; 32x32 cells, 10 steps, every field within
    1e-12 of the oracle, with and without the vacuum term."""
    p = box_params(32, 8, mu=1.0, pmo=pmo)
    s = _tma_solve(nb, p, 6, 21, 10, **HARD)
    assert s.get_tile()[0] == 16
    o = _oracle_solve(p, 6, 21, 10, **HARD)
    a, b = s.get_state(), o.get_state(0)
    for f in range(8):
        assert po.relerr(a[f], b[f]) < FP64_TOL, f
    assert_diag_close(diag_vec(s.analysis()), o.analysis())
    s.close()


@pytest.mark.parametrize("tile", [(16, 32), (8, 7)])
def test_tma_ko4_against_oracle(nb, tile):
    """The TMA kernel with the 4th-difference KO (2 ghost cells, R = 2 queue)
    on 32x32 cells x 162 velocities (the tail kernel runs 160-161), 16- and
    8-row tiles, 10 steps against the oracle."""
    p = box_params(32, 4, mu=1.3, pmo=0.2)
    s = _tma_solve(nb, p, 4, 22, 10, tile=tile, **HARD)
    assert s.get_tile() == tile
    o = _oracle_solve(p, 4, 22, 10, **HARD)
    a, b = s.get_state(), o.get_state(0)
    for f in range(8):
        assert po.relerr(a[f], b[f]) < FP64_TOL, f
    s.close()


def test_tma_ko4_ten_steps_match_reference_on_32_cells(nb):
    """KO4 on the TMA kernel against the reference build's own 10-step state
    (where the reference build is present; the oracle, pinned to it by the CPU
    tests, otherwise)."""
    p = box_params(32, 2)
    s = _tma_solve(nb, p, 4, 9, 10, **PHYS)
    a = s.get_state()
    if po.ref_available(4):
        r = po.RefSim(nn=2, x0=p[0], x1=p[1], z0=p[0], z1=p[1], dx=0.1, dz=0.1, cfl=0.4, ko=0.1, ko_order=4)
        r.fill_init(ipt=1, seed=9, **PHYS)
        r.step(10)
        b = r.get_state(0)
    else:
        b = _oracle_solve(p, 4, 9, 10, **PHYS).get_state(0)
    for f in range(8):
        assert po.relerr(a[f], b[f]) < FP64_TOL, f
    s.close()


def test_fp32_moment_summation_variants(nb):
    """FP32 TMA kernel on 32x32 cells x 642 velocities: summing the
    velocity-moment partials in FP64 (msum 1, the default) leaves the fused
    cell moments within 1e-12 of an FP64 recomputation from the stored FP32
    state; float partials (msum 0) do not reach that (about 1e-7).  Both stay
    within FP32 rounding of the FP64 oracle, and the batch of a member keeps
    its solo bits."""
    p = box_params(32, 8, pmo=0.0)
    o = _oracle_solve(p, 6, 31, 10, **HARD)
    ref = o.get_state(0)
    errs = {}
    for msum in (1, 0):
        s = make(nb, p, 6, precision=nb.FP32, kernel=nb.KERNEL_XTMA)
        assert s.get_moment_sum() == 1
        s.set_moment_sum(msum)
        s.fillInitValue(1, seed=31, **HARD)
        s.step_rk4(10)
        errs[msum] = s.moment_error()
        st = s.get_state()
        for f in range(8):
            assert po.relerr(st[f], ref[f]) < FP32_TOL, (msum, f)
        s.close()
    assert errs[1] < 1e-12, errs
    assert errs[0] > errs[1]


ADV = dict(eps0=1.0, sigma=0.2)  # the reference's advection unit test (Makefile:24-30)


def _adv_params(n, dx=0.02):
    x0, x1 = po.box(n, dx)
    return (x0, x1, dx, 0.25, 0.8, 0.0, 0.0, 2)


@pytest.mark.parametrize("ipt", [10, 20, 30])
def test_advection_initial_data_against_oracle(nb, ipt):
    p = _adv_params(50)
    s = make(nb, p, 4)
    s.fillInitValue(ipt, 0.9, ADV["eps0"], ADV["sigma"], 0.6, 0.5)
    o = _oracle_solve(p, 4, 0, 0, ipt=ipt, **ADV)
    assert po.relerr(s.get_state(), o.get_state(0)) < 1e-15
    np.testing.assert_array_equal(s.G0, np.ones(s.grid.nv))
    s.close()


@pytest.mark.parametrize("n,kernel", [(50, None), (64, 3)])
def test_advection_test_against_oracle(nb, n, kernel):
    """fillInitAdvtest with mu = pmo = 0 (the reference's `make test2d_advec`
    physics, 4th-difference KO 0.8, CFL 0.25), 20 steps: the state within 1e-12
    of the oracle, the I1/I2 integrals of analysis() equal the oracle's, and
    I1 is conserved.  50x50 runs the cp.async/direct kernels (nz % 8 != 0),
    64x64 the TMA kernel."""
    p = _adv_params(n)
    s = make(nb, p, 4, kernel=kernel)
    s.fillInitValue(10, 0.9, ADV["eps0"], ADV["sigma"], 0.6, 0.5)
    d0 = s.analysis()
    s.step_rk4(20)
    d1 = s.analysis()
    o = _oracle_solve(p, 4, 0, 20, ipt=10, **ADV)
    a, b = s.get_state(), o.get_state(0)
    for f in range(8):
        assert po.relerr(a[f], b[f]) < FP64_TOL, f
    np.testing.assert_allclose([d1["I1"], d1["I2"]], o.adv_integrals(), rtol=1e-11)
    assert abs(d1["I1"] - d0["I1"]) < 1e-11 * abs(d0["I1"])
    assert d1["I2"] < d0["I2"]
    s.close()


@pytest.mark.parametrize("kernel", KERNELS)
def test_noc_initial_data_against_oracle(nb, kernel):
    """ipt = 4 ("NOC" Fourier-phase perturbation, seeded phases, every x)
    against the oracle's restatement: the initial state to 1e-15, then 10 steps
    on each stage kernel within 1e-12."""
    p = box_params(64, 2)
    s = make(nb, p, 6)
    s.fillInitValue(4, 0.9, 1e-6, 1.0, 0.6, 0.5, seed=77)
    o = _oracle_solve(p, 6, 77, 0, ipt=4, alpha=0.9, eps0=1e-6, sigma=1.0, lnue=0.6, lnueb=0.5)
    assert po.relerr(s.get_state(), o.get_state(0)) < 1e-15
    np.testing.assert_allclose(s.n_nue0, o.info()["n_nue0"], rtol=1e-12)
    _kernel_ok(nb, s, kernel)
    s.step_rk4(10)
    o.step(10)
    a, b = s.get_state(), o.get_state(0)
    for f in range(8):
        assert po.relerr(a[f], b[f]) < FP64_TOL, f
    s.close()
