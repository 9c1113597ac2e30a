"""FP32 state against the FP64 path: diagnostics error at every output time.

    python -m nuosc_b200.precision_report --size 256 --nn 8 --steps 2000 --every 100 [--hard]

Runs the FP64 solver (parity-checked against the reference) and the FP32
solver (float state and stencil arithmetic, velocity sums in float within a
64-velocity block and in FP64 across blocks, FP64 diagnostics) from the same
seeded initial data, one after the other so that
each can use the whole GPU, and compares the analysis() record at every
output time: |dPee| (surv and survb), |d(|P|-1)| (max and weighted average),
|dM0|.  --hard selects the harder instability case (alpha 1.2, sigma_nubar
0.4, eps 1e-3).  Prints one JSON object with the per-output-time errors, the
maxima, and both precisions' ms/step.
"""
import argparse
import json

KEYS = ("surv", "survb", "maxdP", "avgP", "avgPb", "aM0")


def run(precision, size, nn, steps, every, hard, device=0, seed=20240601, dx=0.05):
    """The production resolution dx = dz = 0.05 (dt = 0.02) on a size x size box;
    coarser grids (dx = 0.2) go unstable within a few hundred steps in the
    reference scheme itself."""
    import torch
    import nuosc_b200 as nb
    L = size * dx / 2
    s = nb.NuOsc(1, 1, nn, 0, 3, 3, -L, L, -L, L, dx, dx, 0.4, 0.1, precision=precision, device=device)
    s.set_mu(1.0)
    s.set_pmo(0.0)
    if hard:
        s.fillInitValue(1, 1.2, 1e-3, 1.0, 0.6, 0.4, seed=seed)
    else:
        s.fillInitValue(1, 0.9, 1e-6, 1.0, 0.6, 0.5, seed=seed)
    stream = torch.cuda.ExternalStream(nb.lib().nuosc_stream(s.handle))
    series = [s.analysis()]
    total_ms, done = 0.0, 0
    for _ in range(steps // every):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s.step_rk4(every)
        e1.record(stream)
        e1.synchronize()
        total_ms += e0.elapsed_time(e1)
        done += every
        try:
            series.append(s.analysis())
        except nb.NuoscError as e:  # the scheme left max||P|-1| < 10 (the reference asserts there)
            if e.code != 4:
                raise
            break
    s.close()
    return series, total_ms / max(1, done)


def report(size, nn, steps, every, hard):
    s64, ms64 = run(0, size, nn, steps, every, hard)
    s32, ms32 = run(1, size, nn, steps, every, hard)
    rows = []
    for a, b in zip(s64, s32):
        rows.append({"phy_time": a["phy_time"], **{"d_" + k: abs(a[k] - b[k]) for k in KEYS},
                     "fp64": {k: a[k] for k in KEYS}})
    worst = {("max_d_" + k): max(r["d_" + k] for r in rows) for k in KEYS}
    return {"size": size, "nv": 10 * nn * nn + 2, "steps": steps, "every": every, "hard": hard,
            "compared_to_step": every * (len(rows) - 1), "fp64_outputs": len(s64), "fp32_outputs": len(s32),
            "ms_per_step_fp64": ms64, "ms_per_step_fp32": ms32, "fp32_speedup": ms64 / ms32,
            "worst": worst, "final": rows[-1], "series": rows}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=256)
    ap.add_argument("--nn", type=int, default=8)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--every", type=int, default=100)
    ap.add_argument("--hard", action="store_true")
    args = ap.parse_args()
    print(json.dumps(report(args.size, args.nn, args.steps, args.every, args.hard)))


if __name__ == "__main__":
    main()
