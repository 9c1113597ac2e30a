"""Serving loop (nuosc_b200.serve).

CPU: the scheduling logic with fake solvers and batches -- every request runs exactly
its step count, analysis records are streamed every `every` steps and at the
last step, admission keeps the resident footprint within the budget and
follows arrival order, oversize requests are rejected, failed solves are
retired (after a blown-up record, or at once by the batch's device-side stop)
with their work counted up to their last passing check, and the one-at-a-time
queue model.
GPU: a mixed FP32/FP64 stream of overlapping requests through the real
batched path; every request's final state and every streamed record equals
the same request run alone with NuOsc.step_rk4 (bit for bit).
"""
import numpy as np
import pytest

from nuosc_b200 import serve


class FakeSolver:
    def __init__(self, req, device=0):
        self.req = req
        self.steps = 0
        self.closed = False

    def step_rk4(self, n):
        assert not self.closed and n >= 1
        self.steps += n
        assert self.steps <= self.req.steps

    @property
    def step_count(self):
        return self.steps

    def synchronize(self):
        pass

    def analysis(self):
        return {"phy_time": self.steps * 0.04, "step": self.steps}

    def close(self):
        self.closed = True


class FakeBatch:
    live = []

    def __init__(self, solvers):
        assert all(not s.closed for s in solvers)
        self.solvers = list(solvers)
        FakeBatch.live.append(self)

    def step_rk4(self, n):
        for s in self.solvers:
            s.step_rk4(n)

    def step_stream(self, n, every):
        recs = []
        for _ in range(n):
            for m, s in enumerate(self.solvers):
                s.step_rk4(1)
                if s.steps % every == 0:
                    recs.append((m, s.steps, s.analysis()))
        return recs

    def collect(self, recs):
        return recs

    def synchronize(self):
        pass

    def close(self):
        FakeBatch.live.remove(self)


def fake_server(budget, every=100, **kw):
    made = {}

    def factory(req, device):
        made[req.rid] = FakeSolver(req)
        return made[req.rid]

    srv = serve.Server(budget_bytes=budget, stream_every=every, solver_factory=factory, batch_factory=FakeBatch,
                       **kw)
    return srv, made


def test_draw_requests_distribution():
    reqs = serve.draw_requests(400, rate=2.0, seed=3)
    assert all(r.nx in (32, 64, 128, 256) and r.nz in (32, 64, 128, 256) for r in reqs)
    assert {r.nn for r in reqs} == {2, 4, 8}
    assert all(100 <= r.steps <= 5000 for r in reqs)
    assert all(0.5 <= r.mu <= 2 and 0.7 <= r.alpha <= 1.3 for r in reqs)
    assert all(0.4 <= r.lnue <= 0.8 and 0.3 <= r.lnueb <= 0.7 and 1e-7 <= r.eps0 <= 1e-3 for r in reqs)
    arr = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(arr) > 0)
    assert 0.6 < np.mean([r.precision == 1 for r in reqs]) < 0.8
    assert 1.5 < len(reqs) / arr[-1] < 2.5  # Poisson rate
    assert serve.draw_requests(5, 1.0, 3)[0] == serve.draw_requests(5, 1.0, 3)[0]  # seeded


def test_footprint_matches_register_layout():
    # 4 registers x 8 fields x cells x padded velocities x element size dominate
    assert serve.footprint_bytes(256, 256, 8, 0) >= 4 * 8 * 256 * 256 * 642 * 8
    assert serve.footprint_bytes(256, 256, 8, 1) >= 4 * 8 * 256 * 256 * 644 * 4
    assert serve.footprint_bytes(32, 32, 2, 1) < serve.footprint_bytes(32, 32, 2, 0)


def test_scheduling_steps_streams_and_budget():
    reqs = serve.draw_requests(40, rate=0.0, seed=5, steps=(7, 450), sizes=(32, 64), nns=(2, 4))
    fp = {r.rid: serve.footprint_bytes(r.nx, r.nz, r.nn, r.precision) for r in reqs}
    budget = 3 * max(fp.values())
    seen = {}
    srv, made = fake_server(budget, every=100, on_diag=lambda rid, step, d: seen.setdefault(rid, []).append(step))
    rep = srv.run(reqs)
    assert rep["served"] == 40 and rep["rejected"] == 0
    assert rep["peak_bytes"] <= budget
    assert 1 < rep["peak_resident"] < 40  # the budget forced queueing
    for r in reqs:
        s = made[r.rid]
        assert s.steps == r.steps and s.closed
        want = [0] + list(range(100, r.steps, 100)) + [r.steps]
        assert seen[r.rid] == sorted(set(want))
    assert not FakeBatch.live


def test_admission_order_and_rejection():
    reqs = serve.draw_requests(6, rate=0.0, seed=9, steps=(10, 20), sizes=(32,), nns=(2,))
    big = serve.Request(rid=99, arrival=0.0, nx=256, nz=256, nn=8, mu=1, alpha=1, lnue=0.6, lnueb=0.5, eps0=1e-6,
                        steps=10, precision=0, seed=1)
    budget = 2.5 * max(serve.footprint_bytes(r.nx, r.nz, r.nn, r.precision) for r in reqs)
    order = []
    srv, made = fake_server(budget, on_diag=lambda rid, step, d: order.append(rid) if step == 0 else None)
    rep = srv.run(reqs + [big])
    assert rep["rejected"] == 1 and 99 not in made
    assert order == [r.rid for r in sorted(reqs, key=lambda r: (r.arrival, r.rid))]


def test_fifo_model():
    reqs = [serve.Request(rid=i, arrival=float(i), nx=32, nz=32, nn=2, mu=1, alpha=1, lnue=0.6, lnueb=0.5,
                          eps0=1e-6, steps=100, precision=0, seed=1) for i in range(3)]
    m = serve.fifo_one_at_a_time(reqs, {0: 2.0, 1: 2.0, 2: 0.5})
    # completions at 2, 4, 4.5 -> latencies 2, 3, 2.5
    assert m["makespan_s"] == pytest.approx(4.5)
    assert m["latency_p50_s"] == pytest.approx(2.5)


def test_record_buffer_pool(monkeypatch):
    """Closed batches hand their page-locked record buffers to a pool that the
    next batch takes from (smallest that fits), so the serving loop frees no
    page-locked memory between quanta; the pool is bounded."""
    import nuosc_b200 as nb

    made, freed = [], []

    class FakeRecords:
        def __init__(self, n):
            self.n, self.used = n, 0
            made.append(self)

        def free(self):
            freed.append(self)

    monkeypatch.setattr(nb, "_PinnedRecords", FakeRecords)
    monkeypatch.setattr(nb, "_REC_POOL", [])
    a = nb._take_records(10)
    assert a.n == nb._REC_MIN and len(made) == 1
    nb._give_records(a)
    assert nb._take_records(100) is a and len(made) == 1  # reused, no new allocation
    big = nb._take_records(5000)
    assert big.n == 5000 and len(made) == 2
    nb._give_records(big)
    nb._give_records(a)
    assert nb._take_records(50) is a  # the smallest that fits
    for k in range(nb._REC_POOL_MAX + 3):
        nb._give_records(FakeRecords(2000 + k))
    assert len(nb._REC_POOL) == nb._REC_POOL_MAX and len(freed) == 4
    assert all(f.n <= min(b.n for b in nb._REC_POOL) for f in freed)


@pytest.mark.gpu
def test_served_results_equal_solo(gpu):
    reqs = serve.draw_requests(12, rate=40.0, seed=11, steps=(30, 260), sizes=(32, 64), nns=(2, 4))
    assert {r.precision for r in reqs} == {0, 1}
    finals, diags = {}, {}
    srv = serve.Server(budget_bytes=150e9, stream_every=50,
                       on_diag=lambda rid, step, d: diags.setdefault(rid, []).append((step, d)),
                       on_complete=lambda rid, s: finals.__setitem__(rid, s.get_state().view(np.uint64)))
    rep = srv.run(reqs)
    # a solve whose state blows up is retired as failed at its first blown-up record
    assert rep["served"] + rep["failed"] == 12 and rep["served"] >= 8 and rep["batch_builds"] >= 2
    assert rep["peak_resident"] > 1  # requests overlapped on the device
    for r in reqs:
        s = serve.make_solver(r)
        want = [(0, serve._analysis(s)[0])]
        done = 0
        for step, _ in diags[r.rid][1:]:
            s.step_rk4(step - done)
            done = step
            want.append((step, serve._analysis(s)[0]))
        assert diags[r.rid] == want
        if r.rid in finals:  # served: every step, and the final state is the solo one
            assert done == r.steps
            assert np.array_equal(finals[r.rid], s.get_state().view(np.uint64))
        else:  # failed: the last record is the first blown-up one
            assert diags[r.rid][-1][1] is None and all(d is not None for _, d in diags[r.rid][:-1])
        s.close()


class BlowUpSolver(FakeSolver):
    """A fake solve whose state blows up at step `bad` (its analysis then
    reports a numeric error, as NuOsc.analysis does for a non-finite state or
    max||P|-1| >= 10)."""
    bad = {}

    def analysis(self):
        b = BlowUpSolver.bad.get(self.req.rid)
        if b is not None and self.steps >= b:
            import nuosc_b200 as nb
            raise nb.NuoscError(nb._lib.ERR_NUMERIC, "blown up")
        return super().analysis()


class BlowUpBatch(FakeBatch):
    def step_stream(self, n, every):
        recs = []
        for _ in range(n):
            for m, s in enumerate(self.solvers):
                s.step_rk4(1)
                if s.steps % every == 0:
                    d, _ = serve._analysis(s)
                    recs.append((m, s.steps, d))
        return recs


def test_blown_up_solves_are_retired_as_failed():
    """A solve whose streamed record reports a blown-up state leaves the GPU
    at the end of that quantum: it runs no more steps, is reported as failed,
    and its cell-steps and latency are not counted as served work."""
    reqs = serve.draw_requests(6, rate=0.0, seed=4, steps=(900, 1000), sizes=(32,), nns=(2,))
    BlowUpSolver.bad = {reqs[1].rid: 250, reqs[4].rid: 100}
    made = {}

    def factory(req, device):
        made[req.rid] = BlowUpSolver(req)
        return made[req.rid]

    srv = serve.Server(budget_bytes=1e12, stream_every=100, solver_factory=factory, batch_factory=BlowUpBatch,
                       quantum_s=1e-9)  # one step per quantum
    rep = srv.run(reqs)
    assert rep["failed"] == 2 and rep["served"] == 4
    for r in reqs:
        s = made[r.rid]
        assert s.closed
        if r.rid == reqs[1].rid:
            assert s.steps == 300  # the record at step 300 is the first blown-up one
        elif r.rid == reqs[4].rid:
            assert s.steps == 100
        else:
            assert s.steps == r.steps
    ok = [r for r in reqs if r.rid not in BlowUpSolver.bad]
    # the failed ones count up to their last good record: steps 200 and 0
    assert rep["cell_steps"] == sum(r.cell_steps for r in ok) + (200 + 0) * 32 * 32 * 42
    assert rep["failed_cell_steps_run"] == (300 + 100) * 32 * 32 * 42
    assert rep["failed_cell_steps_counted"] == 200 * 32 * 32 * 42
    assert not FakeBatch.live


class HaltBatch(BlowUpBatch):
    """A fake batch with the device-side stop (Batch.set_halt/halted): every
    `halt_every` of a member's steps, and at every streamed record, the stop
    test runs on the member's state; a member that fails it stops stepping,
    while its step counter (kept on the solver, as the handle keeps it) goes
    on and its later records repeat its stopped state."""

    def __init__(self, solvers):
        super().__init__(solvers)
        self.halt_every = 0
        for s in self.solvers:
            if not hasattr(s, "counter"):
                s.counter, s.stopped = s.steps, 0

    def set_halt(self, k):
        self.halt_every = k

    def halted(self):
        return [s.stopped for s in self.solvers]

    def step_stream(self, n, every):
        recs = []
        for _ in range(n):
            for m, s in enumerate(self.solvers):
                s.counter += 1
                if not s.stopped:
                    s.step_rk4(1)
                rec = s.counter % every == 0
                if rec or (self.halt_every and s.counter % self.halt_every == 0):
                    d, bad = serve._analysis(s)
                    if bad and self.halt_every and not s.stopped:
                        s.stopped = s.counter
                    if rec:
                        recs.append((m, s.counter, d))
        return recs


def test_device_stop_retires_failed_solves_at_once():
    """With the batch's device-side stop (checks every 10 steps) a failed solve
    stops at its first failing check even in the middle of a long quantum: it
    runs no further steps, its records after the stop are dropped, the failing
    check is its last record, and its steps up to the previous (passing)
    check count as served work."""
    reqs = serve.draw_requests(6, rate=0.0, seed=4, steps=(900, 1000), sizes=(32,), nns=(2,))
    BlowUpSolver.bad = {reqs[1].rid: 250, reqs[4].rid: 100}
    made, diags = {}, {}

    def factory(req, device):
        made[req.rid] = BlowUpSolver(req)
        return made[req.rid]

    srv = serve.Server(budget_bytes=1e12, stream_every=100, solver_factory=factory, batch_factory=HaltBatch,
                       quantum_s=1e9, halt_every=10,
                       on_diag=lambda rid, step, d: diags.setdefault(rid, []).append((step, d)))
    rep = srv.run(reqs)
    assert rep["failed"] == 2 and rep["served"] == 4
    assert made[reqs[1].rid].steps == 250 and made[reqs[4].rid].steps == 100
    assert diags[reqs[1].rid][-1] == (250, None) and all(d is not None for _, d in diags[reqs[1].rid][:-1])
    assert [s for s, _ in diags[reqs[1].rid]] == [0, 100, 200, 250]
    assert diags[reqs[4].rid][-1] == (100, None)
    cells = 32 * 32 * 42
    ok = [r for r in reqs if r.rid not in BlowUpSolver.bad]
    assert rep["cell_steps"] == sum(r.cell_steps for r in ok) + (240 + 90) * cells
    assert rep["failed_cell_steps_run"] == (250 + 100) * cells
    assert rep["failed_cell_steps_counted"] == (240 + 90) * cells
    for r in ok:
        assert made[r.rid].steps == r.steps
    assert not FakeBatch.live


def test_device_stop_counts_work_to_the_last_passing_check():
    """With records every 15 steps and checks every 10, the check grid and the
    record grid interleave (10, 15, 20, 30, 40, 45, ...). A solve that blows
    up at step 41 fails the check at record step 45; the last check it passed
    is the one at step 40, and its work is counted up to there."""
    reqs = serve.draw_requests(3, rate=0.0, seed=5, steps=(300, 300), sizes=(32,), nns=(2,))
    BlowUpSolver.bad = {reqs[0].rid: 41}
    made, diags = {}, {}

    def factory(req, device):
        made[req.rid] = BlowUpSolver(req)
        return made[req.rid]

    srv = serve.Server(budget_bytes=1e12, stream_every=15, solver_factory=factory, batch_factory=HaltBatch,
                       quantum_s=1e9, halt_every=10,
                       on_diag=lambda rid, step, d: diags.setdefault(rid, []).append((step, d)))
    rep = srv.run(reqs)
    assert rep["failed"] == 1 and rep["served"] == 2
    assert made[reqs[0].rid].steps == 45
    assert [s for s, _ in diags[reqs[0].rid]] == [0, 15, 30, 45] and diags[reqs[0].rid][-1] == (45, None)
    cells = 32 * 32 * 42
    assert rep["failed_cell_steps_counted"] == 40 * cells
    assert rep["failed_cell_steps_run"] == 45 * cells
    assert not FakeBatch.live
