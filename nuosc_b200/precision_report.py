"""FP32 state against the FP64 path: diagnostics error at every output time.

    python -m nuosc_b200.precision_report --size 1024 --nn 8 --steps 2000 --every 100 [--hard] [--ko-order 4]

Runs the FP64 solver (parity-checked against the reference) and the FP32
solver (float state and stencil arithmetic; velocity-moment sums as the tile
table says, FP64 by default; FP64 diagnostics) from the same seeded initial
data, one after the other so that each can use the whole GPU, and compares
the analysis() record at every output time: |dPee| (surv and survb),
|d(|P|-1)| (max and weighted average), |dM0|.  --hard selects the harder
instability case (alpha 1.2, sigma_nubar 0.4, eps 1e-3).  --ko-order 4
selects the 4th-difference KO (2 ghosts, the reference's default build):
the reference's 6th-difference KO is anti-dissipative at the grid scale
(its coefficient -ko/(64 dx) times the 6th difference, -64 on that mode,
grows it at the rate ko/dx), so runs with it end when max||P|-1| reaches 10,
while the 4th-difference KO runs stay bounded over 2000 steps.  Prints one
JSON object with the per-output-time errors, the maxima, and both
precisions' ms/step.
"""
import argparse
import json

KEYS = ("surv", "survb", "maxdP", "avgP", "avgPb", "aM0")


def run(precision, size, nn, steps, every, hard, device=0, seed=20240601, dx=0.05, ko_order=6, ko=0.1):
    """The production resolution dx = dz = 0.05 (dt = 0.02) on a size x size box."""
    import torch
    import nuosc_b200 as nb
    L = size * dx / 2
    g = 3 if ko_order == 6 else 2
    s = nb.NuOsc(1, 1, nn, 0, g, g, -L, L, -L, L, dx, dx, 0.4, ko, precision=precision, device=device)
    s.set_mu(1.0)
    s.set_pmo(0.0)
    if hard:
        s.fillInitValue(1, 1.2, 1e-3, 1.0, 0.6, 0.4, seed=seed)
    else:
        s.fillInitValue(1, 0.9, 1e-6, 1.0, 0.6, 0.5, seed=seed)
    stream = torch.cuda.ExternalStream(nb.lib().nuosc_stream(s.handle))
    msum = s.get_moment_sum()
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
    return series, total_ms / max(1, done), msum


def report(size, nn, steps, every, hard, ko_order=6, ko=0.1):
    s64, ms64, _ = run(0, size, nn, steps, every, hard, ko_order=ko_order, ko=ko)
    s32, ms32, msum = run(1, size, nn, steps, every, hard, ko_order=ko_order, ko=ko)
    rows = []
    for a, b in zip(s64, s32):
        rows.append({"phy_time": a["phy_time"], **{"d_" + k: abs(a[k] - b[k]) for k in KEYS},
                     "fp64": {k: a[k] for k in KEYS}})
    worst = {("max_d_" + k): max(r["d_" + k] for r in rows) for k in KEYS}
    return {"size": size, "nv": 10 * nn * nn + 2, "steps": steps, "every": every, "hard": hard,
            "ko_order": ko_order, "ko": ko, "fp32_moment_sum": "fp64" if msum else "float",
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
    ap.add_argument("--ko-order", type=int, default=6, choices=(6, 4))
    ap.add_argument("--ko", type=float, default=0.1)
    args = ap.parse_args()
    print(json.dumps(report(args.size, args.nn, args.steps, args.every, args.hard, args.ko_order, args.ko)))


if __name__ == "__main__":
    main()
