"""Autotuner for the x-march stage kernel's tile shape.

    python -m nuosc_b200.autotune --nn 8 --precision 0 --size 1024 [--write]

For one (velocity count, precision) it times full RK4 steps for every
candidate tile (tz z-rows per CTA in {4, 8, 16}, lx x-planes per CTA) with CUDA
events on the solver's stream, and with --write records the fastest in
nuosc_b200/tiles.txt ("nv precision tz lx" per line), which the library reads
when a handle is created.  The direct kernel is timed too, for reference.
Results are printed as one JSON line.
"""
import argparse
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))
TILES = os.path.join(HERE, "tiles.txt")
DEFAULT_LX = (32, 64, 128, 256, 1 << 20)


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
    s.close()
    best = min((r for r in results if r["kernel"] != "direct"), key=lambda r: r["ms_per_step"])
    return {"nv": 10 * nn * nn + 2, "precision": precision, "size": size, "best": best, "all": results}


def write_table(entries):
    """entries: (nv, precision, tz, lx, kernel kind); kind 2 = cp.async, 3 = TMA x-march."""
    table = {}
    if os.path.exists(TILES):
        for line in open(TILES):
            p = line.split()
            if len(p) >= 4 and not line.startswith("#"):
                table[(int(p[0]), int(p[1]))] = (int(p[2]), int(p[3]), int(p[4]) if len(p) > 4 else 2)
    for nv, prec, tz, lx, kind in entries:
        table[(nv, prec)] = (tz, lx, kind)
    with open(TILES, "w") as f:
        f.write("# nv precision tz lx kernel -- x-march tiles chosen by nuosc_b200/autotune.py "
                "(kernel 2 cp.async, 3 TMA)\n")
        for (nv, prec), (tz, lx, kind) in sorted(table.items()):
            f.write("%d %d %d %d %d\n" % (nv, prec, tz, lx, kind))


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
            entries.append((res["nv"], prec, res["best"]["tz"], res["best"]["lx"], res["best"]["kind"]))
    if args.write:
        write_table(entries)


if __name__ == "__main__":
    main()
