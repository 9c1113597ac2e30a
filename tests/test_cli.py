"""The command-line driver nuosc_b200/nuosc: the reference's main
(nuosc.cpp:17-261) on the C++ facade include/nuosc_b200.hpp.

The 64x64 cells x 162 velocities workload is run with the reference's own
flags (nuosc.cpp:64-139), one extra flag --seed for the seeded perturbation,
and its analysis.dat series (every 10 steps, 100 steps) is compared with the
series the reference build wrote for the same seed (tests/golden/
series_64x64x162.npz), under the tolerances of test_gpu_parity.py.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, golden

pytestmark = pytest.mark.gpu

EXE = os.path.join(ROOT, "nuosc_b200", "nuosc")
DIAG_RTOL = 1e-10
FLAGS = ["--zmax", "3.2", "--dz", "0.1", "--nv", "4", "--cfl", "0.4", "--ko", "0.1", "--mu", "1", "--pmo", "0",
         "--alpha", "0.9", "--lnue", "0.6", "--lnueb", "0.5", "--gz", "3", "--ipt", "1", "--eps0", "1e-6",
         "--sigma", "1", "--ANA_EVERY", "10", "--END_STEP", "100", "--DUMP_EVERY", "50"]


def read_analysis(path):
    rows = [line.split() for line in open(path).read().splitlines() if line and not line.startswith("#")]
    return np.array([[float(x) for x in r] for r in rows])


def test_cli_64x64x162_series_matches_reference(gpu, tmp_path):
    g = golden("series_64x64x162.npz")
    r = subprocess.run([EXE] + FLAGS + ["--seed", str(int(g["seed"]))], cwd=tmp_path, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "[Summ] 1 1 1 64 64 162" in r.stdout, r.stdout
    series = read_analysis(tmp_path / "analysis.dat")
    ref = g["series"]
    assert series.shape == ref.shape
    np.testing.assert_allclose(series[:, [0, 2, 3, 6, 7]], ref[:, [0, 2, 3, 6, 7]], rtol=DIAG_RTOL)
    np.testing.assert_allclose(series[:, 1], ref[:, 1], rtol=1e-4, atol=1e-14)
    np.testing.assert_allclose(series[:, [4, 5]], ref[:, [4, 5]], rtol=1e-4, atol=1e-13)
    np.testing.assert_allclose(series[:, 8], ref[:, 8], atol=1e-11)
    # P3 snapshots at steps 0, 50, 100: [uint t][f64 time][64 x 64 x 17 doubles]
    # (every 162 // 16 = 10th velocity, as the reference's driver slices them)
    for t in (0, 50, 100):
        raw = (tmp_path / ("P3_%06d.bin" % t)).read_bytes()
        assert len(raw) == 4 + 8 + 8 * 64 * 64 * 17
        assert int(np.frombuffer(raw[:4], dtype=np.uint32)[0]) == t
        np.testing.assert_allclose(np.frombuffer(raw[4:12], dtype=np.float64)[0], ref[t // 10, 0], rtol=1e-12)


def test_cli_rejects_two_process_grid(gpu, tmp_path):
    """--np other than 1 1 asks for the reference's MPI decomposition across
    processes, which this driver does not run: it fails with a message."""
    r = subprocess.run([EXE] + FLAGS[:-6] + ["--END_STEP", "1", "--np", "2", "1"], cwd=tmp_path,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode != 0
    assert r.stderr.strip()


ADV_FLAGS = ["--ipt", "10", "--nv", "2", "--gz", "2", "--dz", "0.02", "--zmax", "0.5", "--mu", "0", "--pmo", "0",
             "--eps0", "1", "--sigma", ".2", "--ko", "0.8", "--cfl", "0.25", "--END_STEP_T", ".5",
             "--ANA_EVERY_T", ".1"]


def test_cli_advection_unit_test(gpu, tmp_path):
    """The reference's `make test2d_advec` run (Makefile:24-30, the UNITTEST
    flags with --gz 2) through --ipt 10: 100 steps of pure advection with
    4th-difference KO; the printed I1 (particle number) stays constant and I2
    falls."""
    r = subprocess.run([EXE] + ADV_FLAGS, cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    rows = [line.split() for line in r.stdout.splitlines() if line.startswith("T=") and "I1=" in line]
    assert len(rows) == 6  # t = 0 and every 20 steps
    I1 = np.array([float(x[x.index("I1=") + 1]) for x in rows])
    I2 = np.array([float(x[x.index("I2=") + 1]) for x in rows])
    np.testing.assert_allclose(I1, I1[0], rtol=1e-4)  # printed with 5 digits
    assert np.all(np.diff(I2) < 0)
