"""Autotuner for the x-march stage kernel's tile shape and, in FP32, its
velocity-moment summation.

    python -m nuosc_b200.autotune --nn 8 --precision 0 --size 1024 [--write]

For one (velocity count, precision) it times full RK4 steps for every
candidate tile (tz z-rows per CTA in {4, 8, 16} -- 32 tz threads per CTA --,
lx x-planes per CTA) with CUDA events on the solver's stream.  In FP32 it then
times the best tile with each way of summing the moment partials of a
velocity block (msum 1: FP64 products and sums; 0: float) and measures each
one's summation error (NuOsc.moment_error: the fused cell moments against an
FP64 recomputation from the same stored state); it keeps the fastest whose
error is within MSUM_TOL.  With --write the choice goes to
nuosc_b200/tiles.txt ("nv precision tz lx kernel msum" per line), which the
library reads when a handle is created.  The direct kernel is timed too, for
reference.  Results are printed as one JSON line.

The velocity block of the TMA kernel is not a tuning dimension: it is one
warp's lanes (32 velocities in FP64, 64 in FP32 with two per lane), since the
moment partials are reduced across the lanes of a warp.
"""
import argparse
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))
TILES = os.path.join(HERE, "tiles.txt")
DEFAULT_LX = (32, 64, 128, 256, 1 << 20)
# Largest summation error of the fused FP32 cell moments accepted, relative to
# the largest moment: FP64 accumulation of the stored state's values stays
# near 1e-15 (a compensated float two-sum would have to reach the same bar);
# float partials are near 1e-7 and are rejected.
MSUM_TOL = 1e-12


def time_steps(s, stream, steps, warmup):
    import torch
    s.step_rk4(warmup)
    s.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    s.step_rk4(steps)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / steps


def tune(nn, precision, size, steps=3, warmup=2, lx_list=DEFAULT_LX, device=0, ko_order=6, kinds=(2, 3),
         tz_list=(4, 8, 16)):
    import torch
    import nuosc_b200 as nb
    torch.cuda.set_device(device)
    dx = 51.2 / size
    L = size * dx / 2
    g = 3 if ko_order == 6 else 2
    s = nb.NuOsc(1, 1, nn, 0, g, g, -L, L, -L, L, dx, dx, 0.4, 0.1, precision=precision, device=device)
    s.set_mu(1.0)
    s.set_pmo(0.0)
    s.fillInitValue(1, 0.9, 1e-6, 1.0, 0.6, 0.5, seed=1)
    stream = torch.cuda.ExternalStream(nb.lib().nuosc_stream(s.handle))
    cells = s.grid.nx * s.grid.nz * s.grid.nv
    results = []
    s.set_kernel(nb.KERNEL_DIRECT)
    ms = time_steps(s, stream, steps, warmup)
    results.append({"kernel": "direct", "ms_per_step": ms, "cell_steps_per_s": cells / ms * 1e3})
    for kind, name, tzs in ((nb.KERNEL_XTMA, "xtma", (8, 16)), (nb.KERNEL_XMARCH, "xmarch", (4, 8, 16))):
        if kind not in kinds:
            continue
        s.set_kernel(kind)
        for tz in tzs:
            if tz not in tz_list:
                continue
            if kind == nb.KERNEL_XTMA and s.grid.nz % tz:
                continue
            for lx in lx_list:
                lx = min(lx, s.grid.nx)
                if any(r["kernel"] == name and r.get("tz") == tz and r.get("lx") == lx for r in results):
                    continue
                s.set_tile(tz, lx)
                ms = time_steps(s, stream, steps, warmup)
                results.append({"kernel": name, "kind": kind, "tz": tz, "lx": lx, "ms_per_step": ms,
                                "cell_steps_per_s": cells / ms * 1e3})
    best = min((r for r in results if r["kernel"] != "direct"), key=lambda r: r["ms_per_step"])
    best = dict(best, msum=1)
    msums = []
    if precision == nb.FP32 and best.get("kind") == nb.KERNEL_XTMA:
        s.set_kernel(nb.KERNEL_XTMA)
        s.set_tile(best["tz"], best["lx"])
        for m in (1, 0):
            s.set_moment_sum(m)
            ms = time_steps(s, stream, steps, warmup)
            err = s.moment_error()
            msums.append({"msum": m, "ms_per_step": ms, "moment_error": err, "within_tol": err <= MSUM_TOL})
        ok = [m for m in msums if m["within_tol"]]
        pick = min(ok, key=lambda m: m["ms_per_step"]) if ok else msums[0]
        best = dict(best, msum=pick["msum"], ms_per_step=pick["ms_per_step"],
                    cell_steps_per_s=cells / pick["ms_per_step"] * 1e3)
    s.close()
    return {"nv": 10 * nn * nn + 2, "precision": precision, "size": size, "best": best, "all": results,
            "moment_sum": msums, "msum_tol": MSUM_TOL}


def write_table(entries):
    """entries: (nv, precision, tz, lx, kernel kind, msum); kind 2 = cp.async,
    3 = TMA x-march; msum 1 = FP64 moment sums, 0 = float."""
    table = {}
    if os.path.exists(TILES):
        for line in open(TILES):
            p = line.split()
            if len(p) >= 4 and not line.startswith("#"):
                table[(int(p[0]), int(p[1]))] = (int(p[2]), int(p[3]), int(p[4]) if len(p) > 4 else 2,
                                                 int(p[5]) if len(p) > 5 else 1)
    for nv, prec, tz, lx, kind, msum in entries:
        table[(nv, prec)] = (tz, lx, kind, msum)
    with open(TILES, "w") as f:
        f.write("# nv precision tz lx kernel msum -- x-march tiles chosen by nuosc_b200/autotune.py "
                "(kernel 2 cp.async, 3 TMA; msum 1 FP64 moment sums, 0 float; moment sums within %g)\n" % MSUM_TOL)
        for (nv, prec), (tz, lx, kind, msum) in sorted(table.items()):
            f.write("%d %d %d %d %d %d\n" % (nv, prec, tz, lx, kind, msum))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--nn", type=int, nargs="+", default=[8])
    ap.add_argument("--precision", type=int, nargs="+", default=[0])
    ap.add_argument("--size", type=int, default=1024)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=2)
    ap.add_argument("--lx", type=int, nargs="+", default=list(DEFAULT_LX))
    ap.add_argument("--kinds", type=int, nargs="+", default=[2, 3], help="2 cp.async x-march, 3 TMA x-march")
    ap.add_argument("--tz", type=int, nargs="+", default=[4, 8, 16])
    ap.add_argument("--write", action="store_true")
    args = ap.parse_args()
    entries = []
    for nn in args.nn:
        for prec in args.precision:
            res = tune(nn, prec, args.size, args.steps, args.warmup, args.lx, kinds=tuple(args.kinds),
                       tz_list=tuple(args.tz))
            print(json.dumps(res))
            b = res["best"]
            entries.append((res["nv"], prec, b["tz"], b["lx"], b["kind"], b["msum"]))
    if args.write:
        write_table(entries)


if __name__ == "__main__":
    main()
