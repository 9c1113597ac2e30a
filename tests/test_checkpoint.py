"""Checkpoint and restart (nuosc_save_checkpoint / nuosc_load_checkpoint).

A solve stopped after some steps, saved, loaded into a new handle and
continued gives bit for bit the state of the uninterrupted run -- the file
holds the raw state and the cell moments the last stage kernel accumulated --
on the TMA path in FP64 and FP32 and on the direct path.  A checkpoint of
another grid is refused.
"""
import numpy as np
import pytest

import pyoracle as po

pytestmark = pytest.mark.gpu


def _solver(nb, n=32, nn=4, precision=0, kernel=None, mu=1.3, pmo=0.2):
    x0, x1 = po.box(n, 0.1)
    s = nb.NuOsc(1, 1, nn, 0, 3, 3, x0, x1, x0, x1, 0.1, 0.1, 0.4, 0.1, precision=precision)
    s.set_mu(mu)
    s.set_pmo(pmo)
    if kernel is not None:
        s.set_kernel(kernel)
    return s


@pytest.mark.parametrize("precision,kernel", [(0, 3), (1, 3), (0, 1)])
def test_stop_save_load_continue_is_bit_identical(gpu, tmp_path, precision, kernel):
    import nuosc_b200 as nb
    a = _solver(nb, precision=precision, kernel=kernel)
    a.fillInitValue(1, 1.2, 1e-3, 1.0, 0.6, 0.4, seed=17)
    a.step_rk4(10)
    full = a.get_state()
    d_full = a.analysis()
    a.close()

    b = _solver(nb, precision=precision, kernel=kernel)
    b.fillInitValue(1, 1.2, 1e-3, 1.0, 0.6, 0.4, seed=17)
    b.step_rk4(4)
    path = str(tmp_path / "solve.ck")
    b.save_checkpoint(path)
    b.close()

    c = _solver(nb, precision=precision, kernel=kernel, mu=1.0, pmo=0.0)  # settings come from the file
    c.load_checkpoint(path)
    assert c.step_count == 4
    c.step_rk4(6)
    assert c.step_count == 10
    got = c.get_state()
    assert np.array_equal(got.view(np.uint64), full.view(np.uint64))
    d = c.analysis()
    for k in ("phy_time", "maxdP", "surv", "aM0", "ELNe"):
        assert d[k] == d_full[k], k
    c.close()


def test_checkpoint_of_another_grid_is_refused(gpu, tmp_path):
    import nuosc_b200 as nb
    a = _solver(nb, n=32)
    a.fillInitValue(1, 0.9, 1e-6, 1.0, 0.6, 0.5, seed=1)
    path = str(tmp_path / "a.ck")
    a.save_checkpoint(path)
    a.close()
    for other in (_solver(nb, n=48), _solver(nb, n=32, precision=1), _solver(nb, n=32, nn=2)):
        with pytest.raises(nb.NuoscError) as e:
            other.load_checkpoint(path)
        assert e.value.code == nb._lib.ERR_INVALID
        other.close()
    with pytest.raises(nb.NuoscError):
        _solver(nb).load_checkpoint(str(tmp_path / "missing.ck"))


def test_truncated_checkpoint_leaves_the_handle_unchanged(gpu, tmp_path):
    """A checkpoint file cut short (or with bytes appended) is refused before
    anything is read into the handle: its state, spectra and step count stay
    as they were."""
    import nuosc_b200 as nb
    a = _solver(nb)
    a.fillInitValue(1, 0.9, 1e-3, 1.0, 0.6, 0.5, seed=2)
    a.step_rk4(3)
    path = tmp_path / "a.ck"
    a.save_checkpoint(str(path))
    a.close()
    raw = path.read_bytes()
    b = _solver(nb)
    b.fillInitValue(1, 1.1, 1e-4, 0.8, 0.5, 0.4, seed=5)
    before, d_before = b.get_state(), b.analysis()
    for bad in (raw[:-8], raw + b"\0" * 8):
        cut = tmp_path / "bad.ck"
        cut.write_bytes(bad)
        with pytest.raises(nb.NuoscError) as e:
            b.load_checkpoint(str(cut))
        assert e.value.code == nb._lib.ERR_INVALID
        assert b.step_count == 0
        assert np.array_equal(b.get_state().view(np.uint64), before.view(np.uint64))
        assert b.analysis() == d_before
    b.load_checkpoint(str(path))  # the intact file still loads
    assert b.step_count == 3
    b.close()
