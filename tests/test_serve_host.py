"""CPU tests of the serving loop's host logic (vtib200.serve): the request
generator, the L-BFGS driver (on a quadratic, with the engine replaced by an
exact evaluator) and the stacking of window gradients into the model."""
import numpy as np

import vtib200 as V
import vtib200.serve as SV


def test_requests_follow_the_configured_mix():
    reqs = SV.make_requests(400, rate=20.0, seed=7)
    t = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(t) > 0)
    gaps = np.diff(np.concatenate([[0.0], t]))
    assert abs(gaps.mean() - 1 / 20.0) < 0.01  # Poisson, mean 20 per second
    dims = np.array([r.dim for r in reqs])
    kinds = np.array([r.kind == "gradient" for r in reqs])
    assert 0.4 < (dims == 3).mean() < 0.6 and 0.4 < kinds.mean() < 0.6
    for r in reqs:
        if r.dim == 3:
            nx, ny, nz, nt = r.size
            assert 128 <= nx <= 400 and 128 <= ny <= 400 and 128 <= nz <= 200
        else:
            nx, nz, nt = r.size
            assert 401 <= nx <= 801 and 201 <= nz <= 401
        assert 2000 <= nt <= 4000
    # the same seed gives the same requests
    again = SV.make_requests(400, rate=20.0, seed=7)
    assert [(r.dim, r.kind, r.arrival, r.size) for r in again] == \
           [(r.dim, r.kind, r.arrival, r.size) for r in reqs]


class _Quadratic(SV.FwiDriver):
    """FwiDriver whose 'gradient jobs' are evaluated exactly on the host:
    J(x) = 1/2 (x - x*)^T A (x - x*) split over shots (one window each)."""

    def jobs(self, x):
        return [x.copy() for _ in self.shots]

    def stack(self, results):
        f = sum(r[1] for r in results)
        g = sum(r[0] for r in results)
        return f, g


def _evaluate(x, A, xs, nshot):
    r = x.astype(np.float64) - xs
    f = 0.5 * r @ (A @ r) / nshot
    g = (A @ r / nshot).astype(np.float32)
    return g, f


def test_lbfgs_driver_converges_on_a_quadratic():
    rng = np.random.default_rng(3)
    n = 40
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    A = Q @ np.diag(np.linspace(1.0, 20.0, n)) @ Q.T
    xs = rng.standard_normal(n) + 5.0
    x0 = np.full(n, 5.0, dtype=np.float32)
    shots = [None] * 3
    drv = _Quadratic(None, x0, None, shots, iterations=25, step0=0.5, max_step=1.0,
                     project_stiffness=False)
    jobs = drv.first()
    while jobs is not None:
        jobs = drv.update([_evaluate(j, A, xs, len(shots)) for j in jobs])
    f = np.array(drv.misfits)
    assert f[-1] < 1e-4 * f[0]
    assert np.all(np.diff(f) <= 1e-12 * f[0])  # accepted steps never raise the misfit


def test_lbfgs_step_is_capped_and_nonfinite_trials_are_rejected():
    n = 8
    A = np.eye(n)
    xs = np.full(n, 100.0)
    x0 = np.ones(n, dtype=np.float32)
    drv = _Quadratic(None, x0, None, [None], iterations=2, step0=1000.0, max_step=0.02,
                     project_stiffness=False)
    jobs = drv.first()
    jobs = drv.update([_evaluate(j, A, xs, 1) for j in jobs])
    step = jobs[0] - x0
    assert np.abs(step).max() <= 0.02 * np.abs(x0).max() * (1 + 1e-6)
    # a trial whose misfit is not finite is halved, not accepted
    before = drv.trial.copy()
    nxt = drv.update([(np.zeros(n, dtype=np.float32), float("nan"))])
    assert drv.misfits[-1] == drv.misfits[0] and len(drv.misfits) == 1
    assert np.allclose(nxt[0] - drv.x, 0.5 * (before - drv.x))


def test_lbfgs_first_step_without_step0_moves_by_the_cap():
    """With step0 left at its default the first direction is scaled to the
    max_step cap, so the first trial differs from the starting model."""
    n = 8
    A = np.eye(n)
    xs = np.full(n, 3.0)
    x0 = np.ones(n, dtype=np.float32)
    drv = _Quadratic(None, x0, None, [None], iterations=2, max_step=0.05,
                     project_stiffness=False)
    jobs = drv.first()
    jobs = drv.update([_evaluate(j, A, xs, 1) for j in jobs])
    step = np.abs(jobs[0] - x0).max()
    assert 0 < step <= 0.05 * np.abs(x0).max() * (1 + 1e-6)
    assert np.isclose(step, 0.05, rtol=1e-5)


def test_lbfgs_never_accepts_an_increase():
    """Trials that all raise the misfit: after max_halvings the driver keeps
    the model (the misfit history repeats, never rises) and restarts from
    steepest descent with a shorter step."""
    n = 6
    x0 = np.ones(n, dtype=np.float32)
    drv = _Quadratic(None, x0, None, [None], iterations=3, step0=0.5, max_step=0.1,
                     project_stiffness=False)
    jobs = drv.first()
    jobs = drv.update([(np.ones(n, dtype=np.float32), 1.0)])  # f(x0) = 1
    tried = []
    while jobs is not None:
        tried.append(float(np.abs(jobs[0] - x0).max()))
        jobs = drv.update([(np.ones(n, dtype=np.float32), 2.0)])  # every trial is worse
    assert drv.misfits == [1.0, 1.0, 1.0, 1.0]
    np.testing.assert_array_equal(drv.x, x0)
    assert all(b < a for a, b in zip(tried, tried[1:]))


def test_trial_models_keep_c13_inside_the_stable_range():
    n = 5
    c11 = np.full(n, 4.0, dtype=np.float32)
    c33 = np.full(n, 9.0, dtype=np.float32)
    c13 = np.array([0.0, 5.0, 5.99, 6.5, -7.0], dtype=np.float32)
    drv = SV.FwiDriver(None, np.concatenate([c11, c13, c33]), None, [], iterations=1)
    out = drv.project(np.concatenate([c11, c13, c33]))
    lim = np.float32(0.99) * np.float32(6.0)
    np.testing.assert_array_equal(out[:n], c11)
    np.testing.assert_array_equal(out[2 * n:], c33)
    np.testing.assert_allclose(out[n:2 * n], [0.0, 5.0, lim, lim, -lim], rtol=1e-6)


def test_trial_steps_that_break_the_leapfrog_bound_are_shortened():
    """A step whose trial model would violate dt^2 lambda_max < 4 is halved
    on the host before any gradient is evaluated."""
    g = V.geom3d(12, 10, 8, 10, 2, 10.0, 10.0, 10.0, 1e-3, 2e-3)
    n = 12 * 10 * 8
    v2 = np.float32(3700.0 ** 2)  # dt^2 lambda_max near 3, so doubling breaks the bound
    c = np.concatenate([np.full(n, 1.2 * v2), np.full(n, 1.05 * v2), np.full(n, v2)]).astype(
        np.float32)
    base = V.cfl_number(g, c[:n], c[n:2 * n], c[2 * n:])
    assert 2.5 < base < 3.9
    drv = SV.FwiDriver(g, c, None, [], iterations=1)
    drv.x, drv.p, drv.alpha = c, c.copy(), 1.0  # alpha = 1 would double every stiffness
    t = drv.stable_trial()
    assert drv.alpha < 1.0
    assert V.cfl_number(g, t[:n], t[n:2 * n], t[2 * n:]) < drv.cfl_limit
    drv.p, drv.alpha = 1e-3 * c, 1.0  # a small step is kept as it is
    np.testing.assert_array_equal(drv.stable_trial(), drv.project(c + np.float32(1e-3) * c))
    assert drv.alpha == 1.0


def test_window_gradients_are_stacked_without_their_frames():
    """Window (x0, y0, nx, ny) contributes x in [x0 + pad, x0 + nx - pad) and
    likewise in y, except that a frame lying on the model's edge counts."""
    g = V.geom3d(20, 18, 6, 10, 3, 10.0, 10.0, 10.0, 1e-3, 2e-3)
    # window 0: x [0, 9), y [0, 7); window 1 (reaches the far edges): x [7, 20), y [5, 18)
    wins = [(0, 0, 12, 10), (4, 2, 16, 16)]
    drv = SV.FwiDriver(g, np.zeros(3 * 20 * 18 * 6, dtype=np.float32), None,
                       [(None, None, None, w) for w in wins], iterations=1)
    res = []
    for (x0, y0, wx, wy) in wins:
        res.append((np.ones(1 + 3 * wx * wy * g.nz, dtype=np.float32), 1.5))
    f, full = drv.stack(res)
    assert f == 3.0
    a = full.reshape(3, 6, 18, 20)
    for c in range(3):
        for z in (0, 5):
            expect = {(0, 0): 1, (6, 8): 2, (6, 3): 1, (8, 8): 1, (8, 3): 0, (17, 19): 1,
                      (3, 15): 0}
            for (y, x), v in expect.items():
                assert a[c, z, y, x] == v, (c, z, y, x)


# ------------------------------------------------------------------ failures
# The serving loop's failure handling, driven on the CPU with a stand-in for
# the GPU engine: refused admissions are retried, cancelled requests are
# dropped wherever they are, and an engine failure between ticks (a simulated
# worker death) rebuilds the engine and re-queues what it held.
from types import SimpleNamespace


class _FakeEngine:
    """Engine3d stand-in: at most `slots` jobs at once; a job is finished
    `ticks` engine ticks after admission; its result is (value, 0.0)."""

    made = []

    def __init__(self, slots=2, ticks=3, on_step=None):
        self.slots, self.ticks, self.on_step = slots, ticks, on_step
        self.jobs, self.next = {}, 1
        self.cancelled, self.closed, self.tick = [], False, 0
        _FakeEngine.made.append(self)

    def submit(self, job):
        if len(self.jobs) >= self.slots:
            return None
        jid = self.next
        self.next += 1
        self.jobs[jid] = [job, 0]
        return jid

    def step(self, n):
        self.tick += 1
        if self.on_step:
            self.on_step(self)
        for v in self.jobs.values():
            v[1] += 1
        return sum(v[1] < self.ticks for v in self.jobs.values())

    def poll(self):
        return [j for j, v in self.jobs.items() if v[1] >= self.ticks]

    def result(self, jid):
        job, _ = self.jobs.pop(jid)
        return np.full(3, job.value, dtype=np.float32), 0.0

    def cancel(self, jid):
        self.jobs.pop(jid)
        self.cancelled.append(jid)

    def close(self):
        self.closed = True


def _job(value, n=16):
    return SimpleNamespace(g=SimpleNamespace(nx=n, ny=n, nz=n, nt=10), kind=V.JOB_MODEL,
                           value=value)


def _requests(n3, n2=0):
    reqs = [SV.Request(i, 3, "model", 0.0, (lambda v=i: _job(v))) for i in range(n3)]
    reqs += [SV.Request(n3 + k, 2, "model", 0.0,
                        (lambda v=n3 + k: (lambda ctx: np.full(2, v, np.float32))))
             for k in range(n2)]
    return reqs


def _server(**kw):
    eng = {k: kw.pop(k) for k in ("slots", "ticks", "on_step") if k in kw}
    _FakeEngine.made = []
    return SV.Server(engine_factory=lambda: _FakeEngine(**eng), ctx2=object(), chunk=1, **kw)


def test_refused_admissions_are_retried():
    srv = _server(slots=1, ticks=2, policy="fifo")
    reqs = _requests(4)
    out = srv.run(reqs, t_limit=30.0)
    assert out["done"] == 4 and out["failed"] == 0 and out["cancelled"] == 0
    assert out["refused_admissions"] > 0
    assert all(float(r.result[0][0]) == r.rid for r in reqs)


def test_cancelled_requests_are_dropped_wherever_they_are():
    srv = None

    def on_step(eng):
        if eng.tick == 1:
            srv.cancel(0)  # on the engine by now
            srv.cancel(3)  # still waiting for a slot
            srv.cancel(5)  # a 2D request

    srv = _server(slots=2, ticks=3, on_step=on_step, policy="fifo")
    reqs = _requests(4, 2)
    srv.cancel(4)  # cancelled before it ever runs
    out = srv.run(reqs, t_limit=30.0)
    assert out["cancelled"] + out["done"] == 6
    assert {0, 3, 4} <= {r.rid for r in reqs if r.result is None}
    assert _FakeEngine.made[0].cancelled  # the running job was released on the engine
    for r in reqs:
        if r.result is not None:
            assert float(np.asarray(r.result[0] if r.dim == 3 else r.result)[0]) == r.rid


def test_worker_death_rebuilds_the_engine_and_requeues_its_jobs():
    def fault(tick):
        if tick == 2:
            raise SV.WorkerFault("simulated worker death")

    srv = _server(slots=2, ticks=3, fault=fault, policy="fifo")
    reqs = _requests(5)
    out = srv.run(reqs, t_limit=30.0)
    assert out["done"] == 5 and out["failed"] == 0
    assert out["engine_restarts"] == 1 and out["requeued"] == 2
    assert len(_FakeEngine.made) == 2 and _FakeEngine.made[0].closed
    # every result is the one the request would have had without the fault
    assert all(float(r.result[0][0]) == r.rid for r in reqs)


def test_requests_fail_after_max_fail_attempts():
    def fault(tick):
        raise SV.WorkerFault("the engine keeps failing")

    srv = _server(slots=2, ticks=3, fault=fault, policy="fifo", max_fail=3)
    reqs = _requests(3)
    out = srv.run(reqs, t_limit=30.0)
    assert out["done"] == 0 and out["failed"] == 3
    assert all(isinstance(r.result, SV.WorkerFault) for r in reqs)
