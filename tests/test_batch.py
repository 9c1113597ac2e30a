"""Batched stepping (nuosc_batch_*): every member of a batch must end up with
exactly the bits it gets when stepped alone.

Instances differ in nx, nz, nv (42, 162, 642, 12), mu, pmo (vacuum term on
and off), renormalisation, x-segment length and initial data; each has a twin
built identically and stepped with NuOsc.step_rk4.  States are compared as
raw bit patterns (uint64 view, so even the sign of a zero counts), the
analysis records and phy_time exactly.  The cell spacing 0.125 makes every
box an exact number of cells.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DX = 0.125


@pytest.fixture(scope="module")
def nb(gpu):
    import nuosc_b200
    return nuosc_b200


def build(nb, nx, nz, nn, precision=0, mu=1.0, pmo=0.0, alpha=0.9, eps0=0.1, sigma=0.6, renorm=False,
          lx=None, seed=11, gx=3):
    s = nb.NuOsc(1, 1, nn, 0, gx, gx, -nx * DX / 2, nx * DX / 2, -nz * DX / 2, nz * DX / 2, DX, DX, 0.4, 0.1,
                 precision=precision)
    g = s.grid
    assert (g.nx, g.nz) == (nx, nz)
    s.set_mu(mu)
    s.set_pmo(pmo)
    s.set_renorm(renorm)
    if lx is not None:
        tz, _ = s.get_tile()
        s.set_tile(tz, lx)
    s.fillInitValue(1, alpha, eps0, sigma, 0.6, 0.5, seed=seed)
    return s


def bits(s):
    return s.get_state().view(np.uint64)


def assert_same(a, b):
    assert a.phy_time == b.phy_time
    assert np.array_equal(bits(a), bits(b))
    assert a.analysis() == b.analysis()


SPECS_TZ16 = [dict(nx=48, nz=32, nn=2),
              dict(nx=96, nz=64, nn=4, mu=0.5, pmo=0.1, alpha=1.2, seed=3),
              dict(nx=40, nz=48, nn=8, alpha=0.8, renorm=True, lx=16, seed=5),
              dict(nx=200, nz=32, nn=1, sigma=0.4, seed=9)]
SPECS_TZ8 = [dict(nx=24, nz=16, nn=2, seed=21),
             dict(nx=64, nz=40, nn=4, pmo=0.1, seed=22),
             dict(nx=33, nz=24, nn=8, lx=7, seed=23)]


def run_pair(nb, specs, precision, tz):
    members = [build(nb, precision=precision, **sp) for sp in specs]
    twins = [build(nb, precision=precision, **sp) for sp in specs]
    b = nb.Batch(members)
    try:
        info = b.info()
        assert info["n"] == len(specs) and info["tz"] == tz and info["ctas"] > 0
        # 3 batched steps against 3 solo steps
        b.step_rk4(3)
        b.synchronize()
        for t in twins:
            t.step_rk4(3)
        for m, t in zip(members, twins):
            assert_same(m, t)
        # members continue alone after batched steps
        for m, t in zip(members, twins):
            m.step_rk4(1)
            t.step_rk4(1)
            assert_same(m, t)
        # a setting changed between batch steps is picked up
        members[0].set_mu(0.7)
        twins[0].set_mu(0.7)
        b.step_rk4(2)
        b.synchronize()
        for t in twins:
            t.step_rk4(2)
        for m, t in zip(members, twins):
            assert_same(m, t)
        info = b.info()
        assert info["graph_launches"] == 5
        assert info["kernel_launches"] >= 5 * 8
    finally:
        b.close()
    for s in members + twins:
        s.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_equals_solo_tz16(nb, precision):
    run_pair(nb, SPECS_TZ16, precision, 16)


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_equals_solo_tz8(nb, precision):
    run_pair(nb, SPECS_TZ8, precision, 8)


def test_batch_ko4_equals_solo(nb):
    specs = [dict(nx=48, nz=32, nn=2, gx=2), dict(nx=32, nz=64, nn=4, gx=2, pmo=0.1, seed=4)]
    run_pair(nb, specs, 0, 16)


def test_batch_rejects_bad_membership(nb):
    a = build(nb, 32, 32, 2)
    c = build(nb, 32, 32, 2, precision=1)
    d = build(nb, 32, 20, 2)  # nz % 8 != 0
    try:
        for members, code in (([a, c], nb._lib.ERR_UNSUPPORTED), ([a, a], nb._lib.ERR_INVALID),
                              ([a, d], nb._lib.ERR_UNSUPPORTED)):
            with pytest.raises(nb.NuoscError) as e:
                nb.Batch(members)
            assert e.value.code == code
        b = nb.Batch([a])
        with pytest.raises(nb.NuoscError) as e:
            a.close()  # a member of a live batch is not destroyed
        assert e.value.code == nb._lib.ERR_INVALID
        with pytest.raises(nb.NuoscError) as e:
            nb.Batch([a])  # already in a batch
        assert e.value.code == nb._lib.ERR_INVALID
        b.close()
    finally:
        for s in (a, c, d):
            s.close()


def test_batch_stream_refuses_small_record_buffer(nb):
    """nuosc_batch_step_stream with a record buffer smaller than the records
    the call streams is refused before anything runs: no member steps, and
    the same call with room for its records then matches solo stepping."""
    import ctypes as C
    a, b = build(nb, 32, 32, 2), build(nb, 48, 32, 2, seed=4)
    ta, tb = build(nb, 32, 32, 2), build(nb, 48, 32, 2, seed=4)
    try:
        with nb.Batch([a, b]) as bt:
            recs = (nb._lib.BatchRecord * 4)()
            n = C.c_int(-1)
            rc = nb.lib().nuosc_batch_step_stream(bt.handle, 10, 5, recs, 3, C.byref(n))  # needs 2 x 2 records
            assert rc == nb._lib.ERR_INVALID and n.value == 0
            assert a.step_count == 0 and b.step_count == 0
            rc = nb.lib().nuosc_batch_step_stream(bt.handle, 10, 5, recs, 4, C.byref(n))
            assert rc == nb._lib.OK and n.value == 4
            assert sorted((r.member, r.step) for r in recs) == [(0, 5), (0, 10), (1, 5), (1, 10)]
            bt.synchronize()
        ta.step_rk4(10)
        tb.step_rk4(10)
        assert_same(a, ta)
        assert_same(b, tb)
    finally:
        for s in (a, b, ta, tb):
            s.close()


def off_polarised(nb, s):
    """A state whose polarisation is far off |P| = 1 (emr 20x the diagonal):
    max||P|-1| is about 19, so the reference's stop test fails at once."""
    st = s.get_state()
    st[2] = 20.0 * st[0]
    s.set_state(st)


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_halt_stops_failed_member(nb, precision):
    """nuosc_batch_set_halt: the member that fails the stop test is stopped at
    the first device-side check (step 5) and keeps that state; the others run
    on.  Every member equals its solo run bit for bit: the stopped one after 5
    steps, the others after 20."""
    specs = [dict(nx=48, nz=32, nn=2, seed=31), dict(nx=32, nz=32, nn=4, seed=32),
             dict(nx=64, nz=48, nn=8, seed=33)]
    batch = [build(nb, precision=precision, **sp) for sp in specs]
    solo = [build(nb, precision=precision, **sp) for sp in specs]
    off_polarised(nb, batch[1])
    off_polarised(nb, solo[1])
    with pytest.raises(nb.NuoscError):
        solo[1].analysis()  # the state fails the reference's test from the start
    bt = nb.Batch(batch)
    bt.set_halt(5)
    bt.step_rk4(20)
    bt.synchronize()
    assert bt.halted() == [0, 5, 0]
    bt.close()
    solo[0].step_rk4(20)
    solo[1].step_rk4(5)
    solo[2].step_rk4(20)
    for a, b in zip(batch, solo):
        assert np.array_equal(bits(a), bits(b))
    for s in batch + solo:
        s.close()


def test_batch_without_halt_steps_every_member(nb):
    """Checks off (the default): a failing member is stepped like the others."""
    specs = [dict(nx=48, nz=32, nn=2, seed=41), dict(nx=32, nz=32, nn=2, seed=42)]
    batch = [build(nb, **sp) for sp in specs]
    solo = [build(nb, **sp) for sp in specs]
    off_polarised(nb, batch[1])
    off_polarised(nb, solo[1])
    bt = nb.Batch(batch)
    bt.step_rk4(10)
    bt.synchronize()
    assert bt.halted() == [0, 0]
    bt.close()
    for a, b in zip(batch, solo):
        b.step_rk4(10)
        assert np.array_equal(bits(a), bits(b))
    for s in batch + solo:
        s.close()


def test_batch_halt_stops_renormalised_member(nb):
    """A stopped member with renormalisation on is left alone too (the batch's
    renormalisation and moment passes skip it): a non-finite value planted in
    member 1 fails the stop test at step 5, and member 1 then stays its solo
    state after 5 steps while member 0 (renormalised as well) runs 12."""
    specs = [dict(nx=48, nz=32, nn=2, seed=51, renorm=True), dict(nx=32, nz=32, nn=2, seed=52, renorm=True)]
    batch = [build(nb, **sp) for sp in specs]
    solo = [build(nb, **sp) for sp in specs]
    for s in (batch[1], solo[1]):
        st = s.get_state()
        st[0, 3, 5, 7] = np.nan
        s.set_state(st)
    bt = nb.Batch(batch)
    bt.set_halt(5)
    bt.step_rk4(12)
    bt.synchronize()
    assert bt.halted() == [0, 5]
    bt.close()
    solo[0].step_rk4(12)
    solo[1].step_rk4(5)
    for a, b in zip(batch, solo):
        assert np.array_equal(bits(a), bits(b))
    for s in batch + solo:
        s.close()
