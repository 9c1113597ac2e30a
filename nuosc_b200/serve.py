"""Serving loop: continuous batching of many independent solves on one GPU.

No counterpart in the reference, which runs one NuOsc per process
(nuosc.cpp:171-240).  Requests (a grid, a velocity sphere, physics
parameters, a step count and a precision) arrive over time; the server

  * admits them in arrival order while their HBM footprint fits the budget
    (a request whose footprint exceeds the whole budget is rejected) and
    while the resident work stays below `max_resident_bytes` of state per
    register (1.2 GB: past what saturates the GPU, more residents only
    time-share it -- on 160 mixed requests at 2/s the limit halved the p99
    completion time at the same throughput);
  * keeps every admitted state resident on the device until it completes;
  * packs all resident solves of one precision into one Batch (one
    persistent kernel per RK stage, the step replayed as a CUDA graph) and
    runs the FP32 and FP64 batches on their own streams at the same time;
  * advances in quanta of whole steps that end at the next completion of a
    resident solve or after about `quantum_s` seconds; requests that arrive
    during a quantum are admitted (their solvers built and initial data
    filled) while it runs on the GPU, and join at the next quantum;
  * streams the analysis record (Pee, max||P|-1|, ...) of every solve every
    100 of its steps -- queued on the device between the batch's steps, no
    host synchronisation -- and at its last step;
  * retires a solve as failed when its state blows up (a non-finite value or
    max||P|-1| >= 10, the reference's assert in nuosc_ana.cpp:131): the batch
    applies that test on the device every `halt_every` steps of each member
    (and at every streamed record) and stops a failing member at once -- its
    work is skipped for the rest of the quantum --, and the member leaves its
    batch at the end of the quantum; its steps up to its last passing check
    count as served work (the reference computes them too before it stops),
    the steps after it do not, and it has no completion latency;
  * reports per-request time-to-completion (p50/p99) and the aggregate
    cell-steps/s (nx*nz*nv per RK4 step).

Every solve's result is bit-for-bit what NuOsc.step_rk4 gives it alone (the
batch kernel runs each instance's tiles exactly as its own launch would).

    python -m nuosc_b200.serve --requests 512 --rate 1.5 --seed 7

Request parameters follow a mixed-workload recipe: nx, nz uniform in
{32, 64, 128, 256}, nv in {42, 162, 642} (icosahedron subdivisions 2, 4, 8),
mu ~ U(0.5, 2), alpha ~ U(0.7, 1.3), sigma_nu ~ U(0.4, 0.8), sigma_nubar ~
U(0.3, 0.7), eps amplitude 10^U(-7, -3), steps log-uniform in [100, 5000],
precision FP32 with probability 0.7; cell size 0.1, CFL 0.4, KO 0.1.
"""
import argparse
import json
import math
import time
from dataclasses import dataclass, field

import numpy as np

DX = 0.1
CFL = 0.4
KO = 0.1
STREAM_EVERY = 100
HALT_EVERY = 10  # one analysis pass per 10 steps: about 0.8 % of a step's memory traffic


@dataclass
class Request:
    rid: int
    arrival: float  # seconds after the start of the run
    nx: int
    nz: int
    nn: int  # icosahedron subdivisions: nv = 10 nn^2 + 2
    mu: float
    alpha: float
    lnue: float
    lnueb: float
    eps0: float
    steps: int
    precision: int  # 0 FP64, 1 FP32
    seed: int
    pmo: float = 0.0
    ko_order: int = 6  # 6: the recipe's 6th-difference KO (3 ghosts); 4: 4th difference (2 ghosts)

    @property
    def nv(self):
        return 10 * self.nn * self.nn + 2

    @property
    def cell_steps(self):
        return self.nx * self.nz * self.nv * self.steps


@dataclass
class Record:
    req: Request
    admitted: float = math.nan
    completed: float = math.nan
    diags: list = field(default_factory=list)  # (step, analysis dict or None)
    diverged_at: int = -1  # first streamed step whose analysis reported a blown-up state
    rejected: bool = False
    failed: bool = False  # retired before its last step because its state blew up
    steps_run: int = 0
    last_good: int = 0  # step of the last streamed record, or device-side check, with a passing state

    @property
    def latency(self):
        return self.completed - self.req.arrival


def draw_requests(n, rate, seed, steps=(100, 5000), fp32_frac=0.7, sizes=(32, 64, 128, 256), nns=(2, 4, 8),
                  ko_order=6):
    """n requests with Poisson arrivals at `rate` per second (rate <= 0: all at t=0).
    ko_order 4 gives every request the 4th-difference KO instead of the
    recipe's 6th-difference one, whose anti-dissipative grid-scale term makes
    most long solves blow up (as in the reference)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        if rate > 0:
            t += rng.exponential(1.0 / rate)
        lo, hi = math.log(steps[0]), math.log(steps[1])
        out.append(Request(
            rid=i, arrival=t, nx=int(rng.choice(sizes)), nz=int(rng.choice(sizes)), nn=int(rng.choice(nns)),
            mu=float(rng.uniform(0.5, 2.0)), alpha=float(rng.uniform(0.7, 1.3)),
            lnue=float(rng.uniform(0.4, 0.8)), lnueb=float(rng.uniform(0.3, 0.7)),
            eps0=float(10 ** rng.uniform(-7, -3)), steps=int(round(math.exp(rng.uniform(lo, hi)))),
            precision=1 if rng.uniform() < fp32_frac else 0, seed=int(rng.integers(1, 2 ** 62)),
            ko_order=ko_order))
    return out


def footprint_bytes(nx, nz, nn, precision):
    """Device bytes of one resident solve: 4 state registers, moments, x-march
    moment partials and the small per-handle buffers (as nuosc_create and the
    first step allocate them)."""
    nv = 10 * nn * nn + 2
    esize = 8 if precision == 0 else 4
    align = 16 // esize
    nvs = (nv + align - 1) // align * align
    ncell = nx * nz
    regs = 4 * 8 * ncell * nvs * esize
    nvb = (nvs + 31) // 32
    return regs + ncell * 12 * 8 * (1 + 2 * nvb) + 6 * nvs * 8 + (296 + 1) * 12 * 8 + 256


def register_bytes(req):
    """Bytes of one state register of a request (8 fields x cells x velocities);
    a solve's work per step is proportional to it."""
    return 8 * req.nx * req.nz * req.nv * (8 if req.precision == 0 else 4)


def make_solver(req, device=0):
    """The NuOsc of a request, initial data filled (config-0 recipe: ipt 1,
    eps = eps0 U(-1,1) per cell from the seed)."""
    import nuosc_b200 as nb
    Lx, Lz = req.nx * DX / 2, req.nz * DX / 2
    g = 3 if req.ko_order == 6 else 2
    s = nb.NuOsc(1, 1, req.nn, 0, g, g, -Lx, Lx, -Lz, Lz, DX, DX, CFL, KO, precision=req.precision, device=device)
    g = s.grid
    if (g.nx, g.nz) != (req.nx, req.nz):
        s.close()
        raise ValueError("request %d: grid %dx%d came out as %dx%d" % (req.rid, req.nx, req.nz, g.nx, g.nz))
    s.set_mu(req.mu)
    s.set_pmo(req.pmo)
    s.fillInitValue(1, req.alpha, req.eps0, 1.0, req.lnue, req.lnueb, seed=req.seed)
    return s


def _analysis(s):
    import nuosc_b200 as nb
    try:
        return s.analysis(), False
    except nb.NuoscError as e:
        if e.code != nb._lib.ERR_NUMERIC:
            raise
        return None, True


class Server:
    """Continuous-batching server for NuOsc solves on one GPU.

    on_diag(rid, step, diag)       called for every streamed analysis record
                                   (diag None once the state has blown up)
    on_complete(rid, solver)       called at completion, before the state is freed
    solver_factory(req, device)    builds a request's solver (default make_solver)
    batch_factory(solvers)         builds a batch (default nuosc_b200.Batch);
                                   None steps every solve on its own stream
    """

    def __init__(self, budget_bytes=150e9, device=0, stream_every=STREAM_EVERY, on_diag=None, on_complete=None,
                 solver_factory=None, batch_factory="default", quantum_s=0.25, max_resident_bytes=1.2e9,
                 halt_every=HALT_EVERY):
        self.budget = float(budget_bytes)
        # bytes of one state register summed over the resident solves beyond
        # which admitting more only time-shares a saturated GPU (every
        # resident solve steps once per step of its batch) and stretches
        # everyone's completion time; arrivals then wait in order
        self.max_resident = float(max_resident_bytes)
        self.quantum_s = float(quantum_s)  # target wall time of one quantum (admission granularity)
        self.device = device
        self.every = int(stream_every)
        # steps between the device-side stop tests of a batch member (0: off;
        # failed solves then run to the end of their quantum)
        self.halt_every = int(halt_every)
        self.on_diag = on_diag
        self.on_complete = on_complete
        self.solver_factory = solver_factory or make_solver
        if batch_factory == "default":
            import nuosc_b200 as nb
            batch_factory = nb.Batch
        self.batch_factory = batch_factory

    def run(self, requests):
        reqs = sorted(requests, key=lambda r: (r.arrival, r.rid))
        recs = {r.rid: Record(r) for r in reqs}
        queue = list(reqs)  # arrival order
        active = {}  # rid -> [solver, steps done, footprint]
        batches = {0: None, 1: None}
        members = {0: (), 1: ()}
        used = 0.0
        resident = 0.0  # state bytes of one register, summed over the resident solves
        stats = dict(quanta=0, batch_builds=0, peak_bytes=0.0, peak_resident=0, steps_run=0)
        host = dict(create_s=0.0, build_s=0.0, retire_s=0.0, collect_s=0.0)  # host time per phase
        t0 = time.perf_counter()
        busy = 0.0
        ratio = 1.0  # measured / modelled step time of the last quantum
        inflight = None  # (q, {prec: record buffer}, launch time, modelled step time, solves in it)

        def now():
            return time.perf_counter() - t0

        def stream(rid, step, d):
            rec = recs[rid]
            if d is None and rec.diverged_at < 0:
                rec.diverged_at = step
            if d is not None and rec.diverged_at < 0:
                rec.last_good = step
            rec.diags.append((step, d))
            if self.on_diag:
                self.on_diag(rid, step, d)

        while queue or active or inflight:
            # 1. finish the quantum in flight: streamed records, completions
            if inflight is not None:
                q, bufs, tl, model, ran = inflight
                inflight = None
                for prec in (0, 1):
                    if batches[prec] is not None:
                        batches[prec].synchronize()
                    else:
                        for rid in members[prec]:
                            active[rid][0].synchronize()
                dt_q = time.perf_counter() - tl
                busy += dt_q
                ratio = max(0.05, min(20.0, dt_q / q / model))
                stats["quanta"] += 1
                tc = time.perf_counter()
                halted = {}  # rid -> step at which the batch stopped it on the device
                got = []
                for prec, buf in bufs.items():
                    ids = members[prec]
                    got += [(ids[m], step, d) for m, step, d in batches[prec].collect(buf)]
                    if self.halt_every > 0 and hasattr(batches[prec], "halted"):
                        for m, h in enumerate(batches[prec].halted()):
                            if h > 0:
                                halted[ids[m]] = h
                for rid, step, d in got:
                    if step <= halted.get(rid, step):  # (a stopped solve's later records repeat its stopped state)
                        stream(rid, step, d)
                for rid, h in halted.items():
                    if recs[rid].diverged_at < 0:
                        stream(rid, h, None)  # the failing device-side check is the solve's last record
                    # the previous check passed: the last multiple of halt_every below h, or a later
                    # passing record, which stream() has already counted
                    prev = (h - 1) // self.halt_every * self.halt_every
                    recs[rid].last_good = max(recs[rid].last_good, prev)
                host["collect_s"] += time.perf_counter() - tc
                done = []
                for rid in ran:
                    a = active[rid]
                    a[1] += q
                    ran_steps = min(a[1], halted[rid]) if rid in halted else a[1]
                    stats["steps_run"] += ran_steps - recs[rid].steps_run
                    recs[rid].steps_run = ran_steps
                    if a[1] == recs[rid].req.steps or recs[rid].diverged_at >= 0:
                        done.append(rid)
                for rid in done:
                    s = active[rid][0]
                    req = recs[rid].req
                    if recs[rid].diverged_at < 0 and req.steps % self.every:
                        stream(rid, req.steps, _analysis(s)[0])  # (multiples of `every` were streamed already)
                    # a blown-up state (retired early, or at its last step) is a failed solve
                    recs[rid].failed = recs[rid].diverged_at >= 0
                    recs[rid].completed = now()
                    if self.on_complete and not recs[rid].failed:
                        self.on_complete(rid, s)
                tc = time.perf_counter()
                if done:
                    for prec in (0, 1):  # a solve leaves its batch before it is freed
                        if batches[prec] is not None and set(done) & set(members[prec]):
                            batches[prec].close()
                            batches[prec] = None
                            members[prec] = ()
                    for rid in done:
                        s, _, fp = active.pop(rid)
                        s.close()
                        used -= fp
                        resident -= register_bytes(recs[rid].req)
                host["retire_s"] += time.perf_counter() - tc

            # 2. launch the next quantum on what is resident
            if active:
                tc = time.perf_counter()
                for prec in (0, 1):
                    ids = tuple(sorted(rid for rid, a in active.items() if recs[rid].req.precision == prec))
                    if ids != members[prec]:
                        if batches[prec] is not None:
                            batches[prec].close()
                            batches[prec] = None
                        if ids and self.batch_factory is not None:
                            batches[prec] = self.batch_factory([active[rid][0] for rid in ids])
                            if self.halt_every > 0 and hasattr(batches[prec], "set_halt"):
                                batches[prec].set_halt(self.halt_every)
                            stats["batch_builds"] += 1
                        members[prec] = ids
                host["build_s"] += time.perf_counter() - tc
                model = self._step_model([recs[rid].req for rid in active])
                q = min(recs[rid].req.steps - a[1] for rid, a in active.items())
                q = max(1, min(q, int(self.quantum_s / (model * ratio))))
                bufs = {}
                tl = time.perf_counter()
                for prec in (0, 1):
                    if batches[prec] is not None:
                        bufs[prec] = batches[prec].step_stream(q, self.every)
                    else:
                        for rid in members[prec]:
                            self._solo_quantum(active[rid][0], q, rid, stream)
                inflight = (q, bufs, tl, model, tuple(active))

            # 3. admit arrived requests while the quantum runs: arrival order,
            #    while the footprint fits the budget; they join the next quantum.
            #    With the GPU idle, admit one and go launch it first.
            tc = time.perf_counter()
            while queue and queue[0].arrival <= now() and not (inflight is None and active):
                r = queue[0]
                fp = footprint_bytes(r.nx, r.nz, r.nn, r.precision)
                if fp > self.budget:
                    recs[r.rid].rejected = True
                    queue.pop(0)
                    continue
                if used + fp > self.budget or (active and resident + register_bytes(r) > self.max_resident):
                    break
                queue.pop(0)
                s = self.solver_factory(r, self.device)
                active[r.rid] = [s, 0, fp]
                used += fp
                resident += register_bytes(r)
                recs[r.rid].admitted = now()
                stream(r.rid, 0, _analysis(s)[0])
            host["create_s"] += time.perf_counter() - tc
            stats["peak_bytes"] = max(stats["peak_bytes"], used)
            stats["peak_resident"] = max(stats["peak_resident"], len(active))
            if inflight is None and not active and queue:
                time.sleep(max(0.0, min(queue[0].arrival - now(), 0.05)))
        for b in batches.values():
            if b is not None:
                b.close()
        makespan = now()
        stats.update({k: round(v, 3) for k, v in host.items()})
        return self._report(reqs, recs, makespan, busy, stats)

    @staticmethod
    def _step_model(reqs):
        """Rough seconds per step of the resident set: state bytes moved per
        RK4 step (16 passes of 8 fields) at 4 TB/s, plus launch overhead."""
        b = sum(r.nx * r.nz * r.nv * (1024 if r.precision == 0 else 512) for r in reqs)
        return b / 4e12 + 1e-4

    def _solo_quantum(self, s, q, rid, stream):
        """q steps of one solve on its own stream, analysis every `every` of its steps."""
        done = s.step_count
        left = q
        while left:
            k = min(left, self.every - done % self.every)
            s.step_rk4(k)
            done += k
            left -= k
            if done % self.every == 0:
                stream(rid, done, _analysis(s)[0])

    @staticmethod
    def _report(reqs, recs, makespan, busy, stats):
        """Served = completed every requested step with a finite state.  A failed
        solve (retired on a blown-up record) adds the cell-steps up to its last
        good record to the work done, not the ones after it, and no latency."""
        served = [recs[r.rid] for r in reqs if not recs[r.rid].rejected and not recs[r.rid].failed]
        failed = [recs[r.rid] for r in reqs if recs[r.rid].failed]
        lat = np.array([r.latency for r in served]) if served else np.zeros(1)
        cells = lambda r: r.req.nx * r.req.nz * r.req.nv  # noqa: E731
        good = {r.req.rid: float(cells(r) * r.last_good) for r in failed}
        cs = float(sum(r.req.cell_steps for r in served)) + sum(good.values())
        first = min(r.arrival for r in reqs) if reqs else 0.0
        return {
            "requests": len(reqs), "served": len(served), "rejected": sum(r.rejected for r in recs.values()),
            "failed": len(failed),
            "failed_cell_steps_run": float(sum(cells(r) * r.steps_run for r in failed)),
            "failed_cell_steps_counted": float(sum(good.values())),
            "fp32": sum(r.req.precision == 1 for r in served), "fp64": sum(r.req.precision == 0 for r in served),
            "cell_steps_fp64": float(sum(r.req.cell_steps for r in served if r.req.precision == 0) +
                                     sum(good[r.req.rid] for r in failed if r.req.precision == 0)),
            "cell_steps_fp32": float(sum(r.req.cell_steps for r in served if r.req.precision == 1) +
                                     sum(good[r.req.rid] for r in failed if r.req.precision == 1)),
            "cell_steps": cs, "makespan_s": makespan, "busy_s": busy,
            "cell_steps_per_s": cs / max(1e-9, makespan - first), "cell_steps_per_busy_s": cs / max(1e-9, busy),
            "latency_p50_s": float(np.percentile(lat, 50)), "latency_p99_s": float(np.percentile(lat, 99)),
            "latency_max_s": float(lat.max()), **stats,
        }


def fifo_one_at_a_time(requests, service_s):
    """Completion latencies of the same arrivals served one at a time in
    arrival order, given each request's service time in seconds."""
    t = 0.0
    lat = []
    for r in sorted(requests, key=lambda r: (r.arrival, r.rid)):
        t = max(t, r.arrival) + service_s[r.rid]
        lat.append(t - r.arrival)
    lat = np.array(lat)
    cs = float(sum(r.cell_steps for r in requests))
    first = min(r.arrival for r in requests)
    return {"makespan_s": t, "cell_steps_per_s": cs / max(1e-9, t - first),
            "latency_p50_s": float(np.percentile(lat, 50)), "latency_p99_s": float(np.percentile(lat, 99))}


def solo_fp64_step_times(requests, steps=10, warmup=2, device=0):
    """Measured FP64 step time (s) of the plain single-solve path for every
    distinct (nx, nz, nn, ko_order) among the requests (CUDA events on the
    solver's stream)."""
    import torch
    import nuosc_b200 as nb
    out = {}
    for key in sorted({(r.nx, r.nz, r.nn, r.ko_order) for r in requests}):
        r = Request(rid=-1, arrival=0, nx=key[0], nz=key[1], nn=key[2], mu=1.0, alpha=0.9, lnue=0.6, lnueb=0.5,
                    eps0=1e-6, steps=steps, precision=0, seed=1, ko_order=key[3])
        s = make_solver(r, device)
        st = torch.cuda.ExternalStream(nb.lib().nuosc_stream(s.handle))
        s.step_rk4(warmup)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        s.step_rk4(steps)
        e1.record(st)
        e1.synchronize()
        out[key] = e0.elapsed_time(e1) / 1e3 / steps
        s.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--requests", type=int, default=512)
    ap.add_argument("--rate", type=float, default=1.5, help="Poisson arrival rate, requests per second")
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--budget-gb", type=float, default=150.0)
    ap.add_argument("--max-resident-gb", type=float, default=1.2,
                    help="admit only while one register of the resident solves holds less (0: no limit)")
    ap.add_argument("--min-steps", type=int, default=100)
    ap.add_argument("--max-steps", type=int, default=5000)
    ap.add_argument("--no-baseline", action="store_true", help="skip the one-at-a-time FP64 comparison")
    ap.add_argument("--ko-order", type=int, default=6, choices=(6, 4))
    args = ap.parse_args()
    reqs = draw_requests(args.requests, args.rate, args.seed, steps=(args.min_steps, args.max_steps),
                         ko_order=args.ko_order)
    rep = Server(budget_bytes=args.budget_gb * 1e9,
                 max_resident_bytes=args.max_resident_gb * 1e9 if args.max_resident_gb > 0 else float("inf")).run(reqs)
    rep.update({"rate_per_s": args.rate, "seed": args.seed, "budget_gb": args.budget_gb, "ko_order": args.ko_order,
                "max_resident_gb": args.max_resident_gb,
                "steps_range": [args.min_steps, args.max_steps]})
    if not args.no_baseline:
        t = solo_fp64_step_times(reqs)
        service = {r.rid: t[(r.nx, r.nz, r.nn, r.ko_order)] * r.steps for r in reqs}
        rep["one_at_a_time_fp64"] = {**fifo_one_at_a_time(reqs, service),
                                     "note": "same arrivals served in order on the plain FP64 path; service "
                                             "times from measured per-shape FP64 step times"}
    print(json.dumps(rep))


if __name__ == "__main__":
    main()
