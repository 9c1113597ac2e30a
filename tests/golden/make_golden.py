"""Generate the golden fixtures in tests/golden/ from the reference's own CPU build.

Run from the repository root after `make -C oracle all ref` (which compiles the
reference sources into oracle/_ref/):

    python tests/golden/make_golden.py

Every fixture is produced by the reference's NuOsc (through
oracle/ref_harness/ref_capi.cpp), never by the C restatement, so the
fixtures pin both the oracle and the CUDA path.  Outputs (all .npz):

  quadrature.npz      vx, vy, vz, vw for icosahedron subdivisions nn = 1, 2, 4, 8
  run_ko6.npz         8x8 cells, nv=42: seeded initial state and the state after
  run_ko4.npz         10 RK4 steps, with analysis() before and after
  calrhs_ko6.npz      calRHS of a seeded random state (pmo=0.7, mu=1.3)
  calrhs_ko4.npz      same for the 4th-difference KO branch (pmo=0)
  series_64x64x162.npz  the 64x64 x 162 workload: analysis() every 10 steps
                      for 100 steps and per-field checksums of the final state
  snapshot.npz        bytes of the files addSnapShotAtV / addSnapShotAtXV write
"""
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import pyoracle as po  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

# the physics shared by all run fixtures: alpha 0.9, eps0 1e-6, spectra widths 0.6 / 0.5
PHYS = dict(alpha=0.9, eps0=1e-6, lnue=0.6, lnueb=0.5)


def small_kw(ko_order, n=8, nn=2, dx=0.1, mu=1.0, pmo=0.0, cfl=0.4, ko=0.1):
    x0, x1 = po.box(n, dx)
    return dict(nn=nn, x0=x0, x1=x1, z0=x0, z1=x1, dx=dx, dz=dx, cfl=cfl, ko=ko,
                ko_order=ko_order, mu=mu, pmo=pmo)


def random_state(shape, seed):
    """Well-conditioned random state for calRHS checks (no cancellations)."""
    rng = np.random.default_rng(seed)
    return rng.uniform(-1.0, 1.0, size=(8,) + tuple(shape))


def gen_quadrature():
    out = {}
    for nn in (1, 2, 4, 8):
        r = po.RefSim(**small_kw(6, n=4, nn=nn))
        vx, vy, vz, vw, _, _ = r.velocities()
        out.update({f"vx_{nn}": vx, f"vy_{nn}": vy, f"vz_{nn}": vz, f"vw_{nn}": vw})
        r.close()
    np.savez_compressed(os.path.join(OUT, "quadrature.npz"), **out)


def gen_run(ko_order):
    kw = small_kw(ko_order)
    r = po.RefSim(**kw)
    r.fill_init(ipt=1, seed=1234, **PHYS)
    s0 = r.get_state(0)
    a0 = r.analysis()
    info0 = r.info()
    r.step(10)
    s1 = r.get_state(0)
    a1 = r.analysis()
    _, _, _, _, G0, G0b = r.velocities()
    np.savez_compressed(os.path.join(OUT, f"run_ko{ko_order}.npz"), state0=s0, state10=s1, ana0=a0,
                        ana10=a1, G0=G0, G0b=G0b, n_nue0=np.array(info0["n_nue0"]), seed=1234,
                        params=np.array([kw["x0"], kw["x1"], kw["dx"], kw["cfl"], kw["ko"], kw["mu"],
                                         kw["pmo"], kw["nn"]]))
    r.close()


def gen_calrhs(ko_order, pmo, mu):
    kw = small_kw(ko_order, mu=mu, pmo=pmo)
    r = po.RefSim(**kw)
    nx, nz, nv = r.shape
    inp = random_state((nx, nz, nv), seed=99 + ko_order)
    r.set_state(inp, 0)
    r.calrhs()
    rhs = r.get_state(1)
    np.savez_compressed(os.path.join(OUT, f"calrhs_ko{ko_order}.npz"), inp=inp, rhs=rhs,
                        params=np.array([kw["x0"], kw["x1"], kw["dx"], kw["cfl"], kw["ko"], kw["mu"],
                                         kw["pmo"], kw["nn"]]))
    r.close()


def gen_series():
    x0, x1 = po.box(64, 0.1)
    kw = dict(nn=4, x0=x0, x1=x1, z0=x0, z1=x1, dx=0.1, dz=0.1, cfl=0.4, ko=0.1, ko_order=6, mu=1.0,
              pmo=0.0)
    r = po.RefSim(**kw)
    r.fill_init(ipt=1, seed=2024, **PHYS)
    series = [r.analysis()]
    for _ in range(10):
        r.step(10)
        series.append(r.analysis())
    s = r.get_state(0)
    flat = s.reshape(8, -1)
    sample_idx = np.arange(0, flat.shape[1], 997)
    np.savez_compressed(os.path.join(OUT, "series_64x64x162.npz"), series=np.array(series), seed=2024,
                        fsum=flat.sum(axis=1), fsq=(flat * flat).sum(axis=1),
                        fmax=np.abs(flat).max(axis=1), sample_idx=sample_idx, sample=flat[:, sample_idx])
    r.close()


def gen_snapshot():
    kw = small_kw(6)
    out = {}
    with tempfile.TemporaryDirectory() as d:
        r = po.RefSim(workdir=d, **kw)
        r.fill_init(ipt=1, seed=5, **PHYS)
        r.snapshot_at_v("ee%06d.bin", [0, 21, 41], [0, 2], t=0)
        r.snapshot_at_xv("xv%06d.bin", [1, 4], [3, 7, 40], [4, 6, 3], t=0)
        for name in ("ee%06d.bin" % 0, "ee%06d.bin.meta" % 0, "xv%06d.bin" % 0, "xv%06d.bin.meta" % 0):
            with open(os.path.join(d, name), "rb") as f:
                out[name.replace(".", "_")] = np.frombuffer(f.read(), dtype=np.uint8)
        out["state0"] = r.get_state(0)
        r.close()
    np.savez_compressed(os.path.join(OUT, "snapshot.npz"), **out)


if __name__ == "__main__":
    if not po.ref_available(6) or not po.ref_available(4):
        sys.exit("build the reference first: make -C oracle all ref")
    gen_quadrature()
    gen_run(6)
    gen_run(4)
    gen_calrhs(6, pmo=0.7, mu=1.3)
    gen_calrhs(4, pmo=0.0, mu=1.0)
    gen_series()
    gen_snapshot()
    for f in sorted(os.listdir(OUT)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(OUT, f)))
