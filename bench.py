#!/usr/bin/env python
"""bench.py -- throughput of nuosc's RK4 time step on B200 (cell-steps/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (the production configuration): periodic 2D box of 1024 x 1024 cells
(dx = dz = 0.05, x,z in [-25.6, 25.6)), 642 icosahedral velocities (nn = 8),
FP64 state, 6th-difference Kreiss-Oliger (3 ghosts), CFL 0.4, ko 0.1, mu 1,
alpha 0.9, spectra widths 0.6/0.5, seeded eps = 1e-6 U(-1,1) per cell.
One step = one RK4 step over the whole grid; cell-steps/s = nx*nz*nv per
step / seconds per step.  Each register is 43 GB, far larger than L2, so
no L2 flush is needed between steps.

value    device-timed (CUDA events on the solver's stream), W warm-up steps,
         then K steps, max over ranks; state resident in HBM.
e2e      the same metric through the public C ABI with host buffers: upload
         the state from pinned host memory, K steps each followed by
         analysis() (diagnostics read back), download the final state.
roofline the dominant stage kernel (largest share of the live step time)
         timed with CUDA events on the solver's stream: the state passes that
         stage reads and writes in the 12-pass step (S1 2, S2 4, S3 3, S4 3)
         x 8 fields x 8 B per cell-velocity / mean launch time, against
         the measured HBM copy bandwidth in MEASURED_PEAKS.json.  Step figures
         use the classic RK4 sequence's 1024 B per cell-step (step_frac,
         frac_vs_8tbs) and the 768 B this implementation moves (step_moved_*);
         ncu's DRAM traffic per launch is `traffic` (per step: step_traffic).
N > 1    one independent full-size solve per GPU (the reference's hot path has
         no exchange on one GPU); value = all ranks' cell-steps / max time.
--impl reference   the reference's own CPU build (oracle/_ref, or the C
         oracle where that build is absent) on all host cores, each step one
         RK4 step of a bounded 128 x 128 x 642 sample of the workload (the
         line's config names that sample); the same sample on one thread is
         reported beside (cpu_baseline.one_thread).
extras   (N = 1, skipped with --no-extras) keys "fp32": the same workload
         with FP32 state; "batch": 64 uneven instances per precision in one
         persistent-kernel batch; "serving": a bounded continuous-batching
         run of Poisson-arriving mixed requests with p50/p99 latency.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-steps/s"
# Algorithmic bytes: the classic RK4 stage sequence with registers U, A, Y --
# S1 reads U, writes A and Y (3 passes); S2 and S3 read Y, U and A, write A and
# Y (5 each); S4 reads Y and A, writes U (3) -- 16 passes x 8 fields x
# sizeof(real) per cell-step, the fixed work figure the roofline counts.
BYTES_PER_CELL_STEP = {"f64": 1024, "f32": 512}
# State passes (8 fields each) per stage launch in the 12-pass step of the TMA
# path: S1 reads U, writes Y2; S2 reads Y2 and U, writes Y3 and B; S3 reads Y3
# and U, writes Y4; S4 reads Y4 and B, writes U.
STAGE_PASSES = {"stage_s1": 2, "stage_s2": 4, "stage_s3": 3, "stage_s4": 3}
# The classic sequence's passes for the same stage work (S1 3, S2 5, S3 5, S4 3),
# reported beside as classic_frac
CLASSIC_PASSES = {"stage_s1": 3, "stage_s2": 5, "stage_s3": 5, "stage_s4": 3}
STAGE_NAMES = {"stage_s1": "S1", "stage_s2": "S2", "stage_s3": "S3", "stage_s4": "S4"}
MOVED_BYTES_PER_CELL_STEP = {"f64": 12 * 64, "f32": 12 * 32}


def workload(size, nn, precision):
    dx = 0.05 if size == 1024 else 51.2 / size
    L = size * dx / 2.0
    return dict(n=size, nn=nn, dx=dx, x0=-L, x1=L, precision=precision, cfl=0.4, ko=0.1, mu=1.0, alpha=0.9,
                lnue=0.6, lnueb=0.5, eps0=1e-6, seed=20240601)


def config_of(w, nv, l2_note):
    return {"workload": "RK4 step, %dx%d cells x %d velocities (icosahedron nn=%d), %s state, 6th-difference KO"
                        % (w["n"], w["n"], nv, w["nn"], "FP64" if w["precision"] == 0 else "FP32"),
            "nx": w["n"], "nz": w["n"], "nv": nv, "dx": w["dx"], "cfl": w["cfl"], "ko": w["ko"], "mu": w["mu"],
            "alpha": w["alpha"], "precision": "fp64" if w["precision"] == 0 else "fp32",
            "l2": l2_note, "parallelism": "replicas (one solve per GPU)"}


# ---------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(prefix="nuosc_clocks_", suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        except Exception:
            pass
        finally:
            try:
                os.unlink(self.path)
            except Exception:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------- helpers
def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_per_launch(kernel_key):
    """DRAM bytes per launch of the named kernel from the committed ncu summary, or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return json.load(f).get(kernel_key)
    except Exception:
        return None


def step_traffic(dtype, nx, nv):
    """ncu DRAM bytes of one RK4 step's four stage launches (S1, S2, S3, S4;
    tails and finalize excluded) from the committed per-launch figures, or None."""
    ks = [traffic_per_launch("%s_%s_%d_%d" % (k, dtype, nx, nv)) for k in STAGE_PASSES]
    return float(sum(ks)) if all(k is not None for k in ks) else None


def dist_setup(args=None, backend=None):
    """One process per GPU from the torchrun environment (RANK, LOCAL_RANK,
    WORLD_SIZE, MASTER_*): NCCL when CUDA is present, else gloo (CPU tests)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(cells_per_rank, steps, max_ms, world):
    """Whole-job cell-steps/s of N replicas: all ranks' cell-steps / the slowest rank's time."""
    return world * cells_per_rank * steps / (max_ms / 1e3)


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ---------------------------------------------------------------- CPU arms
def cpu_worker(args):
    """Runs in a subprocess: time RK4 steps of the reference build (or oracle)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    w = workload(args.cpu_size, args.cpu_nn, 0)
    L = w["n"] * 0.1 / 2
    kw = dict(nn=w["nn"], x0=-L, x1=L, z0=-L, z1=L, dx=0.1, dz=0.1, cfl=0.4, ko=0.1, ko_order=6, mu=1.0, pmo=0.0)
    kind = "reference" if po.ref_available(6) else "port"
    sim = po.RefSim(**kw) if kind == "reference" else po.Oracle(**kw)
    sim.fill_init(ipt=1, alpha=0.9, eps0=1e-6, lnue=0.6, lnueb=0.5, seed=w["seed"])
    nx, nz, nv = sim.shape
    for _ in range(args.cpu_warmup):
        sim.step(1)
    times = []
    t_start = time.perf_counter()
    for k in range(args.cpu_steps):
        t0 = time.perf_counter()
        sim.step(1)
        times.append(time.perf_counter() - t0)
        if time.perf_counter() - t_start > args.cpu_budget and k + 1 >= 2:
            break
    total = sum(times)
    print(json.dumps({"kind": kind, "nx": nx, "nz": nz, "nv": nv, "steps": len(times), "seconds": total,
                      "value": nx * nz * nv * len(times) / total, "ms_per_step": 1e3 * total / len(times)}))


def run_cpu(size, nn, steps, warmup, budget, threads=None):
    cores = threads or (len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count())
    env = dict(os.environ, OMP_NUM_THREADS=str(cores), OMP_PROC_BIND="close")
    cmd = [sys.executable, os.path.abspath(__file__), "--cpu-worker", "--cpu-size", str(size), "--cpu-nn", str(nn),
           "--cpu-steps", str(steps), "--cpu-warmup", str(warmup), "--cpu-budget", str(budget)]
    out = subprocess.run(cmd, env=env, stdout=subprocess.PIPE, stderr=subprocess.PIPE, check=True, timeout=1800)
    res = json.loads(out.stdout.decode().strip().splitlines()[-1])
    res["cores"] = cores
    return res


def cpu_baseline_obj(res, one=None):
    o = {"value": res["value"], "unit": METRIC, "cores": res["cores"], "kind": res["kind"],
         "sample": "%dx%d cells x %d velocities, FP64, 6th-difference KO, %d RK4 steps after 1 warm-up, "
                   "OMP threads=%d (%s)" % (res["nx"], res["nz"], res["nv"], res["steps"], res["cores"],
                                            "reference CPU build oracle/_ref" if res["kind"] == "reference"
                                            else "C restatement oracle/")}
    if one is not None:
        o["one_thread"] = {"value": one["value"], "unit": METRIC, "cores": 1, "steps": one["steps"],
                           "ms_per_step": one["ms_per_step"]}
    return o


def one_thread_cpu(args):
    """The same CPU sample on one thread (1 warm-up, at least 2 timed steps)."""
    try:
        return run_cpu(args.cpu_sample, args.nn, 3, 1, budget=args.cpu_seconds_1t, threads=1)
    except Exception:
        return None


def bench_reference(args, world, rank):
    w = workload(args.cpu_sample, args.nn, 0)
    nv = 10 * args.nn * args.nn + 2
    if rank != 0:
        return 0
    res = run_cpu(args.cpu_sample, args.nn, args.steps, max(1, args.warmup), budget=1e9)
    one = one_thread_cpu(args)
    cfg = config_of(w, nv, "n/a (CPU)")
    cfg["workload"] = ("RK4 step of the reference's CPU build on a %dx%d cells x %d velocities sample of the "
                       "%dx%d x %d workload (the full size needs about 283 GB of host memory in the reference's "
                       "layout), FP64, 6th-difference KO, dx 0.1" % (res["nx"], res["nz"], res["nv"], args.size,
                                                                       args.size, nv))
    cfg["dx"] = 0.1
    line = {"metric": METRIC, "value": res["value"], "unit": METRIC, "impl": "reference", "n_gpus": world,
            "steps": res["steps"], "warmup": args.warmup, "ms_per_step": res["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded eps per cell)", "config": cfg,
            "cpu_baseline": cpu_baseline_obj(res, one),
            "e2e": {"value": res["value"], "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------- GPU arm
def bench_ours(args, world, rank, local):
    import numpy as np
    import torch
    import nuosc_b200 as nb

    torch.cuda.set_device(local)
    w = workload(args.size, args.nn, args.precision)
    g = 3
    s = nb.NuOsc(1, 1, w["nn"], 0, g, g, w["x0"], w["x1"], w["x0"], w["x1"], w["dx"], w["dx"], w["cfl"], w["ko"],
                 precision=w["precision"], device=local)
    s.set_mu(w["mu"])
    s.set_pmo(0.0)
    if args.kernel is not None:
        s.set_kernel(args.kernel)
    s.fillInitValue(1, w["alpha"], w["eps0"], 1.0, w["lnue"], w["lnueb"], seed=w["seed"] + rank)
    nx, nz, nv = s.grid.nx, s.grid.nz, s.grid.nv
    cells = nx * nz * nv
    dtype = "f64" if w["precision"] == nb.FP64 else "f32"
    esize = 8 if dtype == "f64" else 4
    stream = torch.cuda.ExternalStream(nb.lib().nuosc_stream(s.handle))

    # warm-up
    s.step_rk4(args.warmup)
    s.synchronize()
    # timed region: K steps, events on the solver's stream, per-kernel events too
    s.set_profiling(True)
    s.get_profile()
    l0 = s.kernel_launches
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        e0.record(stream)
        s.step_rk4(args.steps)
        e1.record(stream)
        e1.synchronize()
    torch.cuda.synchronize()
    barrier(world)
    launches = s.kernel_launches - l0
    prof = s.get_profile()
    s.set_profiling(False)
    ms = max_over_ranks(e0.elapsed_time(e1), world)
    ms_per_step = ms / args.steps
    value = replica_value(cells, args.steps, ms, world)
    diag = s.analysis()

    # dominant kernel: the stage with the largest share of the live step time
    peak, peak_kind = measured_peaks()
    dom = max(STAGE_PASSES, key=lambda k: prof[k][0])
    k_ms, k_n = prof[dom]
    alg_bytes = STAGE_PASSES[dom] * 8 * esize * cells
    launch_s = k_ms / k_n / 1e3 if k_n else None
    achieved = alg_bytes / launch_s / 1e9 if k_n else None
    step_gbs = BYTES_PER_CELL_STEP[dtype] * cells / (ms_per_step / 1e3) / 1e9
    step_moved_gbs = MOVED_BYTES_PER_CELL_STEP[dtype] * cells / (ms_per_step / 1e3) / 1e9
    total_prof = sum(v[0] for v in prof.values()) or 1.0
    stages = {}
    for k in STAGE_PASSES:
        ms_k, n_k = prof[k]
        if n_k:
            b = STAGE_PASSES[k] * 8 * esize * cells
            bc = CLASSIC_PASSES[k] * 8 * esize * cells
            stages[STAGE_NAMES[k]] = {"passes": STAGE_PASSES[k], "mean_launch_ms": ms_k / n_k,
                                      "gbs": b / (ms_k / n_k / 1e3) / 1e9, "frac": b / (ms_k / n_k / 1e3) / 1e9 / peak,
                                      "classic_passes": CLASSIC_PASSES[k],
                                      "classic_frac": bc / (ms_k / n_k / 1e3) / 1e9 / peak}
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak if achieved else None,
                "traffic": traffic_per_launch("%s_%s_%d_%d" % (dom, dtype, nx, nv)),
                "step_traffic": step_traffic(dtype, nx, nv),
                "kernel": "stage %s (%s)" % (STAGE_NAMES[dom], "x-march" if prof["moment_finalize"][1] else "direct"),
                "algorithmic_bytes_per_launch": alg_bytes,
                "per_stage": stages,
                "mean_launch_ms": k_ms / k_n if k_n else None,
                "peak_source": "%s (MEASURED_PEAKS.json hbm_gbs)" % peak_kind if peak_kind == "measured"
                else "fallback 6.65 TB/s",
                "step_bytes_per_cell_step": BYTES_PER_CELL_STEP[dtype], "step_achieved_gbs": step_gbs,
                "step_frac": step_gbs / peak, "frac_vs_8tbs": step_gbs / 8000.0,
                "step_moved_bytes_per_cell_step": MOVED_BYTES_PER_CELL_STEP[dtype],
                "step_moved_gbs": step_moved_gbs, "step_moved_frac": step_moved_gbs / peak,
                "kernel_shares": {k: round(v[0] / total_prof, 4) for k, v in prof.items() if v[1]}}

    # e2e through the C ABI with pinned host buffers
    e2e = None
    if not args.no_e2e:
        host = [torch.empty((nx, nz, nv), dtype=torch.float64, pin_memory=True) for _ in range(8)]
        arrs = [h.numpy() for h in host]
        for f in range(8):
            arrs[f][...] = s.get_field(f)
        barrier(world)
        t0 = time.perf_counter()
        for f in range(8):
            s.set_field(f, arrs[f])
        for _ in range(args.steps):
            s.step_rk4(1)
            s.analysis()
        for f in range(8):
            nb._lib.check(nb.lib().nuosc_get_state(s.handle, 0, f, arrs[f].ctypes.data_as(
                __import__("ctypes").POINTER(__import__("ctypes").c_double)), 0))
        t1 = time.perf_counter()
        barrier(world)
        e2e_s = max_over_ranks(t1 - t0, world)
        state_bytes = 8 * cells * 8
        diag_bytes = 12 * 8
        e2e = {"value": world * cells * args.steps / e2e_s, "unit": METRIC,
               "h2d_bytes_per_step": state_bytes / args.steps,
               "d2h_bytes_per_step": state_bytes / args.steps + diag_bytes,
               "seconds": e2e_s, "pinned": True,
               "note": "upload state from pinned host memory, K x (step_rk4 + analysis), download state"}
        del host, arrs

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            cpu = cpu_baseline_obj(run_cpu(args.cpu_sample, args.nn, 20, 1, budget=args.cpu_seconds),
                                   None if args.no_cpu_1t else one_thread_cpu(args))
        except Exception as ex:  # report, do not fail the GPU number
            cpu = {"value": None, "error": str(ex)[:200]}

    s.close()
    extras = {}
    if rank == 0 and world == 1 and not args.no_extras and w["precision"] == nb.FP64:
        try:
            extras["fp32"] = bench_fp32(args, local, value)
            single = {"f64": value, "f32": extras["fp32"]["value"]}
            extras["batch"] = bench_batch(args, local, single)
            extras["serving"] = bench_serving(args, local, single)
        except Exception as ex:  # report, do not fail the headline number
            extras["extras_error"] = str(ex)[:300]

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": dtype, "data": "synthetic (seeded eps per cell)",
                "config": config_of(w, nv, "inputs larger than L2 (%.1f GB per register)" % (8 * cells * esize / 1e9)),
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk.summary(),
                "gpu_launches": launches, "diag_after": {k: diag[k] for k in ("phy_time", "maxdP", "surv", "aM0")},
                **extras}
        print(json.dumps(line))
    return 0


def bench_fp32(args, local, v64):
    """The FP32 form of the same workload (state and stencil in float; the
    velocity-moment sums as the tile table says -- FP64 -- and the
    diagnostics in FP64): its cell-steps/s and the ratio to FP64."""
    import torch
    import nuosc_b200 as nb
    w = workload(args.size, args.nn, nb.FP32)
    s = nb.NuOsc(1, 1, w["nn"], 0, 3, 3, w["x0"], w["x1"], w["x0"], w["x1"], w["dx"], w["dx"], w["cfl"], w["ko"],
                 precision=nb.FP32, device=local)
    s.set_mu(w["mu"])
    s.set_pmo(0.0)
    s.fillInitValue(1, w["alpha"], w["eps0"], 1.0, w["lnue"], w["lnueb"], seed=w["seed"])
    cells = s.grid.nx * s.grid.nz * s.grid.nv
    st = torch.cuda.ExternalStream(nb.lib().nuosc_stream(s.handle))
    s.step_rk4(args.warmup)
    s.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:  # the FP32 run's own clocks (the ratio compares two timed regions)
        e0.record(st)
        s.step_rk4(args.steps)
        e1.record(st)
        e1.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    s.close()
    v = cells / (ms / 1e3)
    return {"value": v, "unit": METRIC, "ms_per_step": ms, "vs_fp64": v / v64, "steps": args.steps,
            "clocks": clk.summary(),
            "note": "same workload, FP32 state, FP64 moment sums and diagnostics; accuracy vs FP64 in "
                    "profiles/fp32_vs_fp64_1024x642.md"}


def time_large(args, local, precision, gx, steps=3):
    """cell-steps/s of the full-size workload at a given precision and ghost
    width (KO order), W warm-up steps then `steps` timed ones."""
    import torch
    import nuosc_b200 as nb
    w = workload(args.size, args.nn, precision)
    s = nb.NuOsc(1, 1, w["nn"], 0, gx, gx, w["x0"], w["x1"], w["x0"], w["x1"], w["dx"], w["dx"], w["cfl"], w["ko"],
                 precision=precision, device=local)
    s.set_mu(w["mu"])
    s.set_pmo(0.0)
    s.fillInitValue(1, w["alpha"], w["eps0"], 1.0, w["lnue"], w["lnueb"], seed=w["seed"])
    cells = s.grid.nx * s.grid.nz * s.grid.nv
    st = torch.cuda.ExternalStream(nb.lib().nuosc_stream(s.handle))
    s.step_rk4(args.warmup)
    s.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    s.step_rk4(steps)
    e1.record(st)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / steps
    s.close()
    return cells / (ms / 1e3)


def mixed_instances(n, seed, precision):
    """n solves of the mixed-instance recipe: nx, nz from {32, 64, 128, 256},
    nv from {42, 162, 642}, mu, alpha, spectra widths and eps amplitude drawn
    per solve (nuosc_b200.serve.draw_requests)."""
    from nuosc_b200 import serve
    reqs = serve.draw_requests(n, rate=0.0, seed=seed, steps=(100, 100))
    for r in reqs:
        r.precision = precision
    return reqs


def bench_batch(args, local, single):
    """64 uneven instances per precision in one batch (one persistent kernel
    per RK stage, the step a CUDA graph): cell-steps/s and the ratio to the
    single large solve of the same precision."""
    import torch
    import nuosc_b200 as nb
    from nuosc_b200 import serve
    out = {}
    for prec, key in ((nb.FP64, "f64"), (nb.FP32, "f32")):
        reqs = mixed_instances(64, 20240607, prec)
        solvers = [serve.make_solver(r, local) for r in reqs]
        cells = sum(r.nx * r.nz * r.nv for r in reqs)
        b = nb.Batch(solvers)
        st = torch.cuda.ExternalStream(b.stream())
        b.step_rk4(args.warmup)
        b.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        b.step_rk4(args.batch_steps)
        e1.record(st)
        e1.synchronize()
        b.synchronize()
        ms = e0.elapsed_time(e1) / args.batch_steps
        info = b.info()
        b.close()
        for x in solvers:
            x.close()
        v = cells / (ms / 1e3)
        out[key] = {"value": v, "unit": METRIC, "ms_per_step": ms, "vs_single_large_solve": v / single[key],
                    "instances": len(reqs), "cell_velocities": cells, "tiles_per_stage": info["tiles"],
                    "ctas": info["ctas"], "steps": args.batch_steps}
    out["note"] = ("instances drawn with nuosc_b200.serve.draw_requests(seed 20240607): nx, nz in {32,64,128,256}, "
                   "nv in {42,162,642}, mu U(0.5,2), alpha U(0.7,1.3), widths U(0.4,0.8)/U(0.3,0.7), "
                   "eps 10^U(-7,-3); each batched result equals its solo run bit for bit (tests/test_batch.py)")
    return out


def bench_serving(args, local, single):
    """Bounded serving runs of mixed requests (70% FP32) under a 150 GB
    budget with continuous batching: all requests at once (throughput: its
    ratio to the single large solves doing the same cell-steps) and Poisson
    arrivals (p50/p99 completion latency, beside the same arrivals served one
    at a time on the plain FP64 path), with the recipe's 6th-difference KO;
    and all at once again with the 4th-difference KO, under which no request
    blows up (the serving machinery's own throughput)."""
    from nuosc_b200 import serve

    def ref_rate(rep, large=single):  # the large solves' rate for the served FP64/FP32 cell-steps mix
        cs64, cs32 = rep["cell_steps_fp64"], rep["cell_steps_fp32"]
        return (cs64 + cs32) / (cs64 / large["f64"] + cs32 / large["f32"])

    steps = (args.serve_min_steps, args.serve_max_steps)
    sat = serve.draw_requests(args.serve_requests, 0.0, 7, steps=steps)
    rs = serve.Server(budget_bytes=150e9, device=local).run(sat)
    reqs = serve.draw_requests(args.serve_requests, args.serve_rate, 7, steps=steps)
    rp = serve.Server(budget_bytes=150e9, device=local).run(reqs)
    sat4 = serve.draw_requests(args.serve_requests, 0.0, 7, steps=steps, ko_order=4)
    rs4 = serve.Server(budget_bytes=150e9, device=local).run(sat4)
    large4 = {"f64": time_large(args, local, 0, 2), "f32": time_large(args, local, 1, 2)}
    t = serve.solo_fp64_step_times(reqs, device=local)
    one = serve.fifo_one_at_a_time(reqs, {r.rid: t[(r.nx, r.nz, r.nn, r.ko_order)] * r.steps for r in reqs})

    def loop_stats(r):  # device-busy time, quanta, batch rebuilds, host time per server phase
        return {"busy_s": r["busy_s"], "quanta": r["quanta"], "batch_builds": r["batch_builds"],
                "host_s": {k: r[k + "_s"] for k in ("create", "build", "retire", "collect")}}

    return {"requests": len(reqs), "steps_range": list(steps), "budget_gb": 150,
            "saturated": {"cell_steps_per_s": rs["cell_steps_per_s"],
                          "vs_single_large_solve": rs["cell_steps_per_s"] / ref_rate(rs),
                          "makespan_s": rs["makespan_s"], "peak_resident": rs["peak_resident"],
                          "latency_p50_s": rs["latency_p50_s"], "latency_p99_s": rs["latency_p99_s"],
                          **loop_stats(rs)},
            "saturated_ko4": {"cell_steps_per_s": rs4["cell_steps_per_s"],
                              "vs_single_large_solve": rs4["cell_steps_per_s"] / ref_rate(rs4, large4),
                              "single_large_solve_ko4": large4,
                              "served": rs4["served"], "failed": rs4["failed"], "makespan_s": rs4["makespan_s"],
                              "latency_p50_s": rs4["latency_p50_s"], "latency_p99_s": rs4["latency_p99_s"]},
            "poisson": {"rate_per_s": args.serve_rate, "cell_steps_per_s": rp["cell_steps_per_s"],
                        "cell_steps_per_busy_s": rp["cell_steps_per_busy_s"],
                        "latency_p50_s": rp["latency_p50_s"], "latency_p99_s": rp["latency_p99_s"],
                        "makespan_s": rp["makespan_s"], "peak_resident": rp["peak_resident"], **loop_stats(rp),
                        "one_at_a_time_fp64_modelled": {k: one[k] for k in ("cell_steps_per_s", "latency_p50_s",
                                                                            "latency_p99_s", "makespan_s")}},
            "failed": {"saturated": rs["failed"], "poisson": rp["failed"],
                       "saturated_failed_cell_steps_run": rs["failed_cell_steps_run"],
                       "saturated_failed_cell_steps_counted": rs["failed_cell_steps_counted"]},
            "note": "single-large-solve reference = the 1024x1024x642 FP64/FP32 solves timed above, weighted by "
                    "the requests' FP64/FP32 cell-steps; one-at-a-time latencies from measured per-shape FP64 step "
                    "times (modelled: FIFO over measured per-shape step times, no host costs); a request whose "
                    "state fails the reference's stop test (non-finite, or max||P|-1| >= 10; checked on the device "
                    "every 10 steps) is stopped on the device and retired as failed ('failed'): its cell-steps up "
                    "to its last passing check count, the ones after it do not, and it has no latency; "
                    "the 512-request run is in profiles/serving_512_requests.md"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=1024)
    ap.add_argument("--nn", type=int, default=8)
    ap.add_argument("--precision", type=int, default=0, help="0 fp64, 1 fp32")
    ap.add_argument("--kernel", type=int, default=None, help="0 auto, 1 direct, 2 x-march")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-sample", type=int, default=128)
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--cpu-seconds-1t", type=float, default=12.0, help="time budget of the one-thread CPU figure")
    ap.add_argument("--no-cpu-1t", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the FP32, batch and serving sections")
    ap.add_argument("--batch-steps", type=int, default=20)
    ap.add_argument("--serve-requests", type=int, default=64)
    ap.add_argument("--serve-rate", type=float, default=8.0)
    ap.add_argument("--serve-min-steps", type=int, default=20)
    ap.add_argument("--serve-max-steps", type=int, default=500)
    # internal: CPU worker subprocess
    ap.add_argument("--cpu-worker", action="store_true")
    ap.add_argument("--cpu-size", type=int, default=128)
    ap.add_argument("--cpu-nn", type=int, default=8)
    ap.add_argument("--cpu-steps", type=int, default=5)
    ap.add_argument("--cpu-warmup", type=int, default=1)
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    args = ap.parse_args()
    if args.cpu_worker:
        return cpu_worker(args)
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    world, rank, local = dist_setup(args)
    try:
        if args.impl == "reference":
            return bench_reference(args, world, rank)
        return bench_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
