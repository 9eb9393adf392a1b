"""Request loop of the serving workload.

Mixed 2D / 3D modeling and gradient requests arrive over time (seeded
Poisson arrivals). 3D requests go to one `Engine3d` (continuous batching:
admitted between time steps while their device footprint fits the byte
budget, every admitted job advanced by the same launches, state resident on
the device until collected); 2D requests run on a second context (its own
CUDA stream) in a worker thread, so their kernels overlap the 3D launches on
the device. An optional FWI driver interleaves L-BFGS iterations of gradient
requests on a 3D model. The loop reports per-request latency (arrival to
result on the host) as p50 / p99 and requests per second.
"""
from __future__ import annotations

import queue
import threading
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from . import (JOB_GRADIENT, JOB_MODEL, OPT_FULL_STEPS, Context, Engine3d, Plan3d, VtiError,
               cfl_number, geom3d, get_boundary, objFuncGradient_f, synthetic_f, vepsdel_to_cij)
from . import synth as S


@dataclass
class Request:
    rid: int
    dim: int            # 2 or 3
    kind: str           # "model" or "gradient"
    arrival: float      # seconds after the start
    make: object        # callable building the job (3D) or the call arguments (2D)
    size: tuple = ()
    t_admit: float = -1.0
    t_done: float = -1.0
    result: object = None
    tag: object = None  # caller's label (FWI shot)

    @property
    def latency(self):
        return self.t_done - self.arrival


def _layered3d(nx, ny, nz, d, seed):
    z = np.arange(nz) * d
    v1, e1, d1 = S.layered(z, S.interfaces_for(nz * d, seed=seed))
    shape = (nz, ny, nx)
    v = np.broadcast_to(v1[:, None, None], shape).reshape(-1).astype(np.float32)
    e = np.broadcast_to(e1[:, None, None], shape).reshape(-1).astype(np.float32)
    dl = np.broadcast_to(d1[:, None, None], shape).reshape(-1).astype(np.float32)
    return vepsdel_to_cij(v, e, dl)


def job3d(kind, nx, ny, nz, nt, freq, seed, d=12.5, dt=1e-3, npad=20, rec_step=4):
    """A 3D request: layered VTI model, source at the centre, receivers on a
    grid 25 m below the top; gradient requests get zero observed traces (the
    residual is the modeled data; the work does not depend on the values).
    The pad is at most a quarter of the smallest dimension."""
    npad = min(npad, min(nx, ny, nz) // 4)
    o = -npad * d
    g = geom3d(nx, ny, nz, nt, npad, d, d, d, dt, 4e-3, ox=o, oy=o, oz=o)
    c11, c13, c33 = _layered3d(nx, ny, nz, d, seed)
    w = S.ricker(nt, dt, freq)
    rx = np.arange(npad, nx - npad, rec_step)
    ry = np.arange(npad, ny - npad, rec_step)
    RX, RY = np.meshgrid(rx, ry, indexing="xy")
    rec = np.zeros((RX.size, 4), dtype=np.float32)
    rec[:, 0] = RX.reshape(-1) * d + o + 0.25 * d
    rec[:, 1] = RY.reshape(-1) * d + o + 0.25 * d
    rec[:, 2] = (npad + 2) * d + o + 0.25 * d
    rec[:, 3] = 1
    so = np.array([nx // 2 * d + o + 0.25 * d, ny // 2 * d + o + 0.25 * d,
                   (npad + 2) * d + o + 0.25 * d, RX.size, 0], dtype=np.float32)
    nnt = (nt - 1) // 4 + 1
    if kind == "model":
        return Engine3d.make_job(JOB_MODEL, g, c11, c13, c33, w, so, rec)
    return Engine3d.make_job(JOB_GRADIENT, g, c11, c13, c33, w, so, rec,
                             dobs=np.zeros(nnt * RX.size, dtype=np.float32), seed=seed)


def call2d(kind, nz, nx, nt, freq, seed, npad=30):
    """A 2D request: the layered survey of lib/vti-fwi-2d's conventions."""
    s = S.survey2d(nx=nx, nz=nz, nt=nt, npad=npad, freq=freq, seed=seed)
    g = s.geom()
    if kind == "model":
        return lambda ctx: synthetic_f(ctx, g, s.c11, s.c13, s.c33, s.wavelet, s.sloc, s.rloc,
                                       s.taper)
    ratio = int(round(g.rate / g.dt))
    data = np.zeros(((nt - 1) // ratio + 1, s.rloc.size // 2), dtype=np.float32)
    return lambda ctx: objFuncGradient_f(ctx, g, data, s.c11, s.c13, s.c33, s.wavelet, s.sloc,
                                         s.rloc, s.taper)


def make_requests(n, rate=20.0, seed=7, size3d=((128, 128, 128), (400, 400, 200)),
                  size2d=((201, 401), (401, 801)), nt=(2000, 4000), freq=(10.0, 15.0)):
    """n requests with Poisson arrivals (mean `rate` per second): half 2D, half
    3D, half modeling, half gradient; grid sizes, nt and the Ricker frequency
    drawn uniformly in the given ranges (3D: nx, ny, nz; 2D: nz, nx)."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=n))
    out = []
    for i in range(n):
        dim = 3 if rng.random() < 0.5 else 2
        kind = "gradient" if rng.random() < 0.5 else "model"
        steps = int(rng.integers(nt[0], nt[1] + 1))
        f = float(rng.uniform(*freq))
        if dim == 3:
            (a, b, c), (A, B, Cc) = size3d
            nx, ny, nz = (int(rng.integers(a, A + 1)), int(rng.integers(b, B + 1)),
                          int(rng.integers(c, Cc + 1)))
            mk = (lambda k=kind, x=nx, y=ny, z=nz, s=steps, ff=f, sd=seed * 1000 + i:
                  job3d(k, x, y, z, s, ff, sd))
            size = (nx, ny, nz, steps)
        else:
            (a, b), (A, B) = size2d
            nz, nx = int(rng.integers(a, A + 1)), int(rng.integers(b, B + 1))
            mk = (lambda k=kind, z=nz, x=nx, s=steps, ff=f, sd=seed * 1000 + i:
                  call2d(k, z, x, s, ff, sd))
            size = (nx, nz, steps)
        out.append(Request(i, dim, kind, float(t[i]), mk, size))
    return out


@dataclass
class FwiDriver:
    """L-BFGS on a 3D model (c11, c13, c33 stacked) with gradients from
    gradient requests on windows of the model, one request per shot and
    iteration; the next iteration is submitted when the last gradient of the
    current one has arrived. A step that raises the misfit (or whose misfit
    is not finite) is halved and re-evaluated, at most `max_halvings` times;
    if none lowers the misfit the iteration keeps the current model and
    clears the L-BFGS memory (the next direction is steepest descent), so
    the accepted misfits never increase. A step never changes a stiffness by
    more than `max_step` of the largest one, and with `project_stiffness`
    every trial model keeps |c13| <= 0.99 sqrt(c11 c33) (beyond it the VTI
    system is not hyperbolic and wavefields grow without bound) and a step
    whose trial model breaks the leapfrog bound (dt^2 lambda_max >=
    `cfl_limit`, vti3d_cfl_number) is halved before it is evaluated."""
    g: object
    model: np.ndarray
    wavelet: np.ndarray
    shots: list          # (souloc[5], recloc, dobs, window) per shot
    iterations: int
    memory: int = 3
    max_halvings: int = 2
    max_step: float = 0.02
    misfits: list = field(default_factory=list)
    step0: float = 0.0
    project_stiffness: bool = True
    cfl_limit: float = 3.9

    def __post_init__(self):
        self.s_hist, self.y_hist = [], []
        self.x = np.array(self.model, dtype=np.float32)
        self.it = 0
        self.g_cur = None
        self.f_cur = None
        self.trial = None
        self.halvings = 0
        self.restarts = 0  # consecutive directions without a decrease

    def jobs(self, x):
        """One gradient job per shot on its window of model x; the random
        boundary of each window is a fixed host-generated multiplier (the
        same for every iteration and for the plain evaluation)."""
        g, n = self.g, self.g.nx * self.g.ny * self.g.nz
        if not hasattr(self, "_r2"):
            self._r2 = []
            for k, (_, _, _, (x0, y0, wx, wy)) in enumerate(self.shots):
                r = S.random_boundary(np.ones(wx * wy * g.nz, dtype=np.float32), wx, wy, g.nz,
                                      g.npad, seed=101 + k)
                self._r2.append((r * r).astype(np.float32))
        out = []
        for k, (so, rec, dobs, (x0, y0, wx, wy)) in enumerate(self.shots):
            sub = geom3d(wx, wy, g.nz, g.nt, g.npad, g.dx, g.dy, g.dz, g.dt, g.sampling_rate,
                         ox=g.ox + x0 * g.dx, oy=g.oy + y0 * g.dy, oz=g.oz)
            c = [x[i * n:(i + 1) * n].astype(np.float32).reshape(g.nz, g.ny, g.nx)
                 [:, y0:y0 + wy, x0:x0 + wx].reshape(-1) for i in range(3)]
            randb = np.concatenate([get_boundary(ci * self._r2[k], wx, wy, g.nz, g.npad)
                                    for ci in c])
            out.append(Engine3d.make_job(JOB_GRADIENT, sub, *c, self.wavelet, so, rec,
                                         dobs=dobs, randb=randb))
        return out

    def run_plain(self, ctx):
        """The same iterations with the plain form: vti3d_plan_gradient of one
        shot at a time. Returns the misfit history."""
        jobs = self.first()
        while jobs is not None:
            jobs = self.update([plain_gradient(ctx, j) for j in jobs])
        return self.misfits

    def stack(self, results):
        g, n = self.g, self.g.nx * self.g.ny * self.g.nz
        full = np.zeros((3, g.nz, g.ny, g.nx), dtype=np.float32)
        f = 0.0
        for (fg, mis), (_, _, _, (x0, y0, wx, wy)) in zip(results, self.shots):
            f += mis
            ns = wx * wy * g.nz
            xl, xh = (0 if x0 == 0 else g.npad), (wx if x0 + wx == g.nx else wx - g.npad)
            yl, yh = (0 if y0 == 0 else g.npad), (wy if y0 + wy == g.ny else wy - g.npad)
            for c in range(3):
                a = fg[1 + c * ns:1 + (c + 1) * ns].reshape(g.nz, wy, wx)
                full[c, :, y0 + yl:y0 + yh, x0 + xl:x0 + xh] += a[:, yl:yh, xl:xh]
        return f, full.reshape(-1)

    def direction(self, grad):
        """L-BFGS two-loop recursion; vectors in FP32, dot products in FP64."""
        q = grad.copy()
        al = []
        for s, y in reversed(list(zip(self.s_hist, self.y_hist))):
            a = _dot(s, q) / _dot(y, s)
            al.append(a)
            q -= np.float32(a) * y
        if self.y_hist:
            s, y = self.s_hist[-1], self.y_hist[-1]
            q *= np.float32(_dot(s, y) / _dot(y, y))
        else:
            # no curvature pair yet: the first step's largest change is step0,
            # or (step0 <= 0) the max_step cap relative to the largest stiffness
            s0 = self.step0 if self.step0 > 0 else self.max_step * float(np.abs(self.x).max())
            q *= np.float32(s0 / max(float(np.abs(q).max()), 1e-300))
        for (s, y), a in zip(zip(self.s_hist, self.y_hist), reversed(al)):
            b = _dot(y, q) / _dot(y, s)
            q += np.float32(a - b) * s
        return -q

    def project(self, x):
        """Trial model clipped to |c13| <= 0.99 sqrt(c11 c33) (x = c11, c13, c33)."""
        if not self.project_stiffness:
            return x
        n = x.size // 3
        c11, c13, c33 = x[:n], x[n:2 * n], x[2 * n:]
        lim = (np.float32(0.99) * np.sqrt(np.maximum(c11, 0) * np.maximum(c33, 0))).astype(
            np.float32)
        out = x.copy()
        out[n:2 * n] = np.clip(c13, -lim, lim)
        return out

    def stable_trial(self):
        """x + alpha p projected; alpha halved (at most 30 times) while the
        trial model breaks the leapfrog bound."""
        for _ in range(30):
            t = self.project(self.x + np.float32(self.alpha) * self.p)
            if not self.project_stiffness or self.g is None:
                return t
            n = t.size // 3
            if cfl_number(self.g, t[:n], t[n:2 * n], t[2 * n:]) < self.cfl_limit:
                return t
            self.alpha *= 0.5
        return t

    def first(self):
        self.trial = self.x
        return self.jobs(self.x)

    def update(self, results):
        """Results of the submitted jobs in; the next jobs out (None: done)."""
        f, grad = self.stack(results)
        if not np.isfinite(f) and self.f_cur is not None:
            f = np.inf  # a trial model outside the stable range: halve the step
        if self.f_cur is not None and not f < self.f_cur and self.halvings >= self.max_halvings:
            # no decrease along this direction: keep the model, restart L-BFGS
            # with steepest descent, its step shortened 8x for each restart in a row
            self.s_hist, self.y_hist = [], []
            self.it += 1
            self.misfits.append(self.f_cur)
            self.halvings = 0
            self.restarts += 1
            if self.it >= self.iterations:
                return None
            self.p = self.direction(self.g_cur)
            cap = self.max_step * float(np.abs(self.x).max())
            pmax = float(np.abs(self.p).max())
            self.alpha = (min(1.0, cap / pmax) if pmax > 0 else 1.0) * 0.125 ** self.restarts
            self.trial = self.stable_trial()
            return self.jobs(self.trial)
        if self.f_cur is None or f < self.f_cur:
            if self.f_cur is not None:
                s, y = self.trial - self.x, grad - self.g_cur
                if _dot(s, y) > 0:
                    self.s_hist.append(s)
                    self.y_hist.append(y)
                    self.s_hist, self.y_hist = self.s_hist[-self.memory:], self.y_hist[-self.memory:]
                self.it += 1
            self.x, self.f_cur, self.g_cur = self.trial, f, grad
            self.misfits.append(f)
            self.halvings = 0
            self.restarts = 0
            if self.it >= self.iterations:
                return None
            self.p = self.direction(grad)
            # at most max_step (relative to the largest stiffness) per iteration
            cap = self.max_step * float(np.abs(self.x).max())
            pmax = float(np.abs(self.p).max())
            self.alpha = min(1.0, cap / pmax) if pmax > 0 else 1.0
        else:
            self.alpha *= 0.5
            self.halvings += 1
        self.trial = self.stable_trial()
        return self.jobs(self.trial)


def _dot(a, b):
    return float(np.einsum("i,i->", a, b, dtype=np.float64))


def plain_gradient(ctx, job):
    """A gradient job through vti3d_plan_gradient (VTI_OPT_FULL_STEPS) on the
    job's grid: (fgcij, misfit)."""
    c11, c13, c33, w, so, rec, dobs, randb = job._keep
    p = Plan3d(ctx, job.g, OPT_FULL_STEPS)
    try:
        p.set_model(c11, c13, c33, randb=randb)
        p.set_wavelet(w)
        p.set_receivers(rec)
        return p.gradient(so, [0], dobs)
    finally:
        p.close()


def _points(job):
    return job.g.nx * job.g.ny * job.g.nz


def _work(r):
    """Estimated device work of a 3D request: points x time steps x the
    wavefield-pair updates per step (1 modeling, 4 gradient)."""
    j = r._job
    return _points(j) * j.g.nt * (4 if j.kind == JOB_GRADIENT else 1)


def _summary(res):
    """(sum, L2 norm, misfit) of a result, for callers that keep no arrays."""
    arrs = [a for a in (res if isinstance(res, tuple) else (res,)) if isinstance(a, np.ndarray)]
    mis = [float(a) for a in (res if isinstance(res, tuple) else ()) if isinstance(a, float)]
    return (sum(float(np.sum(a, dtype=np.float64)) for a in arrs),
            sum(float(np.linalg.norm(a.reshape(-1).astype(np.float64))) for a in arrs),
            mis[-1] if mis else None)


class WorkerFault(RuntimeError):
    """The engine failed between ticks (raised by a fault hook to simulate a
    worker death, or standing for a device error reported by the engine)."""


# Attempts per request before it is reported failed: the reference's job farm
# resubmits a failed job up to MAX_FAIL = 5 times (lib/vti-fwi-3d/gpu/cluster.h:4,
# objFuncGradient3d_f.cu:60-64).
MAX_FAIL = 5


class Server:
    """Continuous-batching request loop on one GPU.

    Failure handling (all on the host, between ticks): a request can be
    cancelled at any time (`cancel`); an admission the engine refuses for
    lack of memory is retried on later ticks; if the engine fails (an error
    from a step, or a `fault` hook raising WorkerFault before a tick), the
    engine is torn down and rebuilt and every request it held is queued again
    from its start, up to `max_fail` attempts, after which it is reported
    failed."""

    def __init__(self, device=0, max_bytes=64 << 30, chunk=16, keep_results=True, log=None,
                 policy="sjf", max_active_points=24_000_000, engine_factory=None, ctx2=None,
                 fault=None, max_fail=MAX_FAIL):
        """policy "sjf": waiting 3D jobs are admitted shortest (grid points x
        time steps x passes) first, and only while the grid points of the
        jobs in flight stay within max_active_points (a larger job runs
        alone): a launch that already fills the GPU gains nothing from more
        jobs, which would only share its time. policy "fifo": arrival order,
        no cap (memory budget only). engine_factory / ctx2 replace the GPU
        engine and the 2D context (tests drive the loop with stand-ins);
        fault(tick) is called before every engine step that has jobs in flight,
        with the number of that step (1, 2, ...)."""
        self._own = engine_factory is None
        if self._own:
            self.ctx3 = Context(device)
            self.ctx2 = Context(device)
            engine_factory = lambda: Engine3d(self.ctx3, max_bytes)  # noqa: E731
        else:
            self.ctx2 = ctx2
        self._factory = engine_factory
        self.engine = engine_factory()
        self.chunk = chunk
        self.keep_results = keep_results
        self.log = log
        self.policy = policy
        self.max_active_points = max_active_points
        self.fault = fault
        self.max_fail = max_fail
        self._lock = threading.Lock()
        self._cancel = set()

    def _log(self, msg):
        if self.log:
            self.log(msg)

    def cancel(self, rid):
        """Cancels request `rid` (thread-safe): it is dropped wherever it is
        (not yet arrived, waiting, on the engine, or queued for the 2D
        worker); a request already done is unaffected."""
        with self._lock:
            self._cancel.add(rid)

    def _cancelled(self, rid):
        with self._lock:
            return rid in self._cancel

    def close(self):
        self.engine.close()
        if self._own:
            self.ctx3.close()
            self.ctx2.close()

    def run(self, requests, fwi: FwiDriver | None = None, t_limit=3600.0):
        t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0  # noqa: E731
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        waiting = deque()
        q2 = queue.Queue()
        inflight = {}
        done = []
        fwi_reqs = []
        cancelled, failed = [], []
        counts = {"requeued": 0, "engine_restarts": 0, "refused_admissions": 0}
        tick = 0

        ready = {}  # request id -> prepared 3D job (built off the stepping thread)
        q3 = queue.Queue()

        def prep():
            while True:
                r = q3.get()
                if r is None:
                    return
                ready[id(r)] = r.make()

        tp = threading.Thread(target=prep, daemon=True)
        tp.start()

        def worker():
            while True:
                r = q2.get()
                if r is None:
                    return
                if self._cancelled(r.rid):
                    r.t_done = now()
                    cancelled.append(r)
                    continue
                r.t_admit = now()
                res = r.make()(self.ctx2)
                r.result = res if self.keep_results else _summary(res)
                r.t_done = now()
                done.append(r)
                self._log(f"request {r.rid} (2D {r.kind}) done at {r.t_done:.2f} s")

        th = threading.Thread(target=worker, daemon=True)
        th.start()

        def submit_fwi(jobs):
            for k, j in enumerate(jobs):
                r = Request(-1, 3, "gradient", now(), lambda jj=j: jj, tag=k)
                r._job = j
                fwi_reqs.append(r)
                waiting.append(r)

        if fwi is not None:
            submit_fwi(fwi.first())
        fwi_batch = {}
        n2 = sum(r.dim == 2 for r in requests)

        def drop_cancelled():
            with self._lock:
                cset = set(self._cancel)
            if not cset:
                return
            for lst in (pending, waiting):
                for r in [r for r in lst if r.rid >= 0 and r.rid in cset]:
                    lst.remove(r)
                    r.t_done = now()
                    cancelled.append(r)
            for jid in [j for j, r in inflight.items() if r.rid >= 0 and r.rid in cset]:
                r = inflight.pop(jid)
                self.engine.cancel(jid)
                r.t_done = now()
                cancelled.append(r)

        def worker_death(err):
            """Tear the engine down and rebuild it; its requests start again."""
            counts["engine_restarts"] += 1
            self._log(f"engine failed at tick {tick}: {err}; restarting it with "
                      f"{len(inflight)} request(s) re-queued")
            try:
                self.engine.close()
            except Exception as e:  # the old engine may be unusable
                self._log(f"closing the failed engine: {e}")
            self.engine = self._factory()
            for r in sorted(inflight.values(), key=lambda x: x.t_admit, reverse=True):
                r.attempts = getattr(r, "attempts", 0) + 1
                if r.attempts >= self.max_fail:
                    r.t_done = now()
                    r.result = err
                    failed.append(r)
                else:
                    counts["requeued"] += 1
                    waiting.appendleft(r)
            inflight.clear()

        while now() < t_limit:
            drop_cancelled()
            t = now()
            while pending and pending[0].arrival <= t:
                r = pending.popleft()
                if r.dim == 2:
                    q2.put(r)
                else:
                    q3.put(r)
                    waiting.append(r)
            refused = False
            for r in waiting:
                if not hasattr(r, "_job") and id(r) in ready:
                    r._job = ready.pop(id(r))
            if self.policy == "sjf":
                order = sorted((r for r in waiting if hasattr(r, "_job")), key=_work)
            else:
                order = []
                for r in waiting:  # arrival order up to the first job still being built
                    if not hasattr(r, "_job"):
                        break
                    order.append(r)
            active_pts = sum(_points(x._job) for x in inflight.values())
            for r in order:
                pts = _points(r._job)
                if (self.policy == "sjf" and inflight and
                        active_pts + pts > self.max_active_points):
                    break
                jid = self.engine.submit(r._job)
                if jid is None:
                    # retried on a later tick; with nothing in flight the job
                    # can never fit the budget
                    refused = not inflight
                    counts["refused_admissions"] += 1
                    break
                waiting.remove(r)
                r.t_admit = now()
                inflight[jid] = r
                active_pts += pts
            try:
                if inflight:
                    tick += 1
                    if self.fault is not None:
                        self.fault(tick)
                active = self.engine.step(self.chunk) if inflight else 0
                finished = [(jid, self.engine.result(jid)) for jid in self.engine.poll()]
            except (WorkerFault, VtiError) as err:
                worker_death(err)
                continue
            for jid, res in finished:
                r = inflight[jid]
                del inflight[jid]
                r.t_done = now()
                del r._job
                if r.rid >= 0:
                    r.result = res if self.keep_results else _summary(res)
                    done.append(r)
                    self._log(f"request {r.rid} ({r.dim}D {r.kind}) done at {r.t_done:.2f} s")
                else:
                    fwi_batch[r.tag] = res
            if fwi is not None and fwi_batch and len(fwi_batch) == len(fwi.shots):
                nxt = fwi.update([fwi_batch[k] for k in range(len(fwi.shots))])
                fwi_batch = {}
                self._log(f"FWI evaluation done at {now():.2f} s, misfit {fwi.misfits[-1]:.6g}, "
                          f"iteration {fwi.it}")
                if nxt is not None:
                    submit_fwi(nxt)
                else:
                    fwi = None
            n_done = sum(r.rid >= 0 for r in done + cancelled + failed)
            if n_done == len(requests) and fwi is None and not inflight and not waiting:
                break
            if not active and not inflight:
                if refused:
                    raise RuntimeError("request larger than the engine's memory budget")
                if waiting:
                    time.sleep(0.001)  # a job is being built
                    continue
                if pending:
                    time.sleep(max(0.0, min(pending[0].arrival - now(), 0.05)))
                elif n_done < len(requests):
                    time.sleep(0.002)
        q2.put(None)
        q3.put(None)
        th.join()
        tp.join()
        lat = np.array([r.latency for r in done if r.rid >= 0])
        first = min(r.arrival for r in requests) if requests else 0.0
        last = max((r.t_done for r in done), default=first)
        return {
            "requests": len(requests), "done": int(len(lat)), "n2d": n2,
            "n3d": len(requests) - n2,
            "p50_s": float(np.percentile(lat, 50)) if len(lat) else None,
            "p99_s": float(np.percentile(lat, 99)) if len(lat) else None,
            "makespan_s": last - first,
            "requests_per_s": len(lat) / max(last - first, 1e-9),
            "fwi_requests": len(fwi_reqs),
            "cancelled": sum(r.rid >= 0 for r in cancelled),
            "failed": sum(r.rid >= 0 for r in failed),
            **counts,
        }
