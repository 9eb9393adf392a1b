"""Benchmark: 3D VTI adjoint gradient (fwd + adjoint) throughput on B200.

Workload (one "step" = one L2-misfit gradient evaluation of one shot, the
three passes of objFuncGradientCij3d_f): 400 x 400 x 200 grid at 12.5 m
(40-cell pad inside), dt = 1 ms, nt = 3000 (all 2999 levels), 12 Hz Ricker,
200 x 200 receivers at 25 m, 4 ms trace sampling; layered VTI model with a
Gaussian random-field perturbation; observed data from the true model, the
gradient at the smoothed (250 m) model. Synthetic, seeded inputs.

Metric: grid-point updates per second (Gpts/s): 4 wavefield-pair updates per
time level (pass 1 forward, pass 2 forward, pass 3 source reconstruction and
adjoint) x nx*ny*nz points x levels, summed over all ranks.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Under torchrun each rank models its own shot (weak scaling); the gradients
are summed with one NCCL all-reduce per step. `value` is device-resident
throughput; `e2e` goes through the host-buffer C-ABI entry point
(vti3d_gradient_cij) with pinned host inputs and outputs.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "thesis-source-code_b200"))
# the oracle (test infrastructure) is used only by the cpu_baseline, error and
# reference legs below, never inside the timed GPU region
sys.path.insert(0, str(ROOT / "oracle"))


def _configs():
    import vtib200.synth as S
    return {
        # name: survey3d kwargs
        "gradient400": dict(S.GRADIENT400),
        "small": dict(S.GRADIENT400, nx=128, ny=128, nz=96, nt=402, npad=16, smooth_m=100.0),
        # profiling case: every volume (34 MB) x 14 inputs exceeds the 126 MB L2
        "mid": dict(S.GRADIENT400, nx=256, ny=256, nz=128, nt=130, npad=24, smooth_m=100.0),
    }


CONFIGS = _configs()
BWD_BYTES_PER_POINT = 84  # 14 reads + 7 writes of FP32 per point (fused backward)
FWD_BYTES_PER_POINT = 36  # 7 reads + 2 writes


def peaks():
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        d = json.loads(f.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, device):
        self.device, self.rows, self.proc = device, [], None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4)
                          if len(r) > 4 + k and r[4 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def make_inputs(cfg, rank, nt=None):
    import vtib200.synth as S
    kw = dict(CONFIGS[cfg])
    if nt:
        kw["nt"] = nt
    return S.gradient_inputs(kw, rank)


def levels(g, flags):
    return g.nt - 1 if flags & 1 else 1 + 64 * ((g.nt - 2) // 64)


GRADIENT_METRIC = "3D VTI fwd+adjoint gradient throughput (grid-point updates/s)"
CPU_SAMPLE_NT = 66   # time samples of one CPU sample of the gradient (65 levels)
CHECK_NT = 130       # time samples of the full-grid check against the FP64 oracle


def gradient_config(cfg, s, M, nrec):
    """The workload description both arms print (identical object)."""
    return {"workload": f"3D VTI L2-misfit gradient, {cfg}: {s.nx}x{s.ny}x{s.nz} grid "
                        f"(pad {s.npad}), nt={s.nt}, {M} levels, {nrec} receivers, "
                        "1 shot per GPU",
            "grid": [s.nx, s.ny, s.nz], "nt": s.nt, "levels": M, "receivers": nrec,
            "shots_per_gpu": 1,
            "points": "nx*ny*nz per wavefield-pair update, 4 updates per level (pass 1, "
                      "pass 2, pass 3 source and adjoint); the 4-cell x/y frame the scheme "
                      "never updates is 4% of them",
            "l2": "wavefields (133 MB each) larger than L2 (126 MB); no flush"}


def shortened(s, nt):
    """The same survey over its first nt time samples (the Ricker wavelet is
    evaluated per sample, so it is the first nt values)."""
    import dataclasses
    return dataclasses.replace(s, nt=nt, wavelet=np.ascontiguousarray(s.wavelet[:nt]))


def first_samples(dobs, nrec, nnt_full, nnt):
    """Trace-major traces ([receiver][sample]) cut to their first nnt samples."""
    return np.ascontiguousarray(np.asarray(dobs, dtype=np.float32).reshape(nrec, nnt_full)
                                [:, :nnt]).reshape(-1)


class OracleGeom:
    """Geometry attributes the oracle reads (no library needed)."""

    def __init__(self, s):
        self.nx, self.ny, self.nz, self.nt, self.npad = s.nx, s.ny, s.nz, s.nt, s.npad
        self.ox = self.oy = self.oz = s.o
        self.ot = 0.0
        self.dx = self.dy = self.dz = s.d
        self.dt, self.sampling_rate = s.dt, s.rate


def oracle_gradient_sample(s, cstart, padb, randb, dobs):
    """One timed CPU sample: the FP32 oracle's whole three-pass gradient
    (REFERENCE mode, all levels) of survey s on its full grid, all host
    threads. Returns (Gpts/s counted as the GPU arm counts, seconds)."""
    import oracle as O
    g = OracleGeom(s)
    t0 = time.perf_counter()
    O.gradient3d(g, cstart, padb, randb, s.wavelet, s.souloc, [0], s.recloc, dobs,
                 dtype=np.float32, full_steps=True)
    sec = time.perf_counter() - t0
    M = s.nt - 1
    return 4.0 * (M - 1) * s.nxyz / sec / 1e9, sec


def cpu_sample_desc(s, threads):
    return (f"the FP32 oracle's whole gradient (pass 1 with traces and misfit, pass 2, "
            f"pass 3) on the full {s.nx}x{s.ny}x{s.nz} grid over the first {s.nt} time "
            f"samples ({s.nt - 1} levels) of the same shot, {threads} OpenMP threads")


def oracle_errors(ctx, s, cstart, ctrue, padb, randb, nt):
    """GPU vs the FP64 oracle on the full grid over the first nt samples:
    modeled traces, misfit and the three gradients through the host-buffer
    C ABI (VTI_OPT_FULL_STEPS); the FP32 oracle's own error against FP64 is
    the FP32 noise level for comparison."""
    import oracle as O
    import vtib200 as V
    t0 = time.perf_counter()
    sh = shortened(s, nt)
    g = sh.geom()
    n = sh.nxyz
    flags = V.OPT_FULL_STEPS
    sp = lambda c: (c[:n], c[n:2 * n], c[2 * n:])  # noqa: E731
    dobs = V.modelDataCij3d_f(ctx, g, sh.souloc, [0], sh.recloc, sh.wavelet, *sp(ctrue),
                              flags=flags)
    dmod = V.modelDataCij3d_f(ctx, g, sh.souloc, [0], sh.recloc, sh.wavelet, *sp(cstart),
                              flags=flags)
    fg, mis = V.objFuncGradientCij3d_f(ctx, g, sh.souloc, [0], sh.recloc, sh.wavelet, cstart,
                                       padb, randb, dobs, flags=flags)
    og = OracleGeom(sh)
    o64, m64 = O.gradient3d(og, cstart, padb, randb, sh.wavelet, sh.souloc, [0], sh.recloc,
                            dobs, dtype=np.float64, full_steps=True, want_modeled=True)
    o32, m32 = O.gradient3d(og, cstart, padb, randb, sh.wavelet, sh.souloc, [0], sh.recloc,
                            dobs, dtype=np.float32, full_steps=True, want_modeled=True)

    def rl2(a, b):
        a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
        return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))

    part = lambda f, k: f[1 + k * n:1 + (k + 1) * n]  # noqa: E731
    return {"nt": nt, "levels": nt - 1, "grid": [sh.nx, sh.ny, sh.nz],
            "api": "vti3d_model_data_cij + vti3d_gradient_cij (host buffers)",
            "traces_rel_l2": rl2(dmod, m64), "misfit_rel": abs(mis - o64[0]) / o64[0],
            "gradient_rel_l2": [rl2(part(fg, k), part(o64, k)) for k in range(3)],
            "fp32_oracle_gradient_rel_l2": [rl2(part(o32, k), part(o64, k)) for k in range(3)],
            "fp32_oracle_traces_rel_l2": rl2(m32, m64),
            "tolerance": {"traces": 1e-5, "misfit": 1e-5, "gradient": 1e-4},
            "seconds": round(time.perf_counter() - t0, 1)}


def run_b200(args):
    import torch
    import torch.distributed as dist
    import vtib200 as V

    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device(
            "cuda", local))
    s, cstart, ctrue, padb, randb = make_inputs(args.config, rank)
    g = s.geom()
    flags = V.OPT_FULL_STEPS
    n = s.nxyz
    ctx = V.Context(local)
    plan = V.Plan3d(ctx, g, flags)
    plan.set_wavelet(s.wavelet)
    plan.set_receivers(s.recloc)
    nrec = s.recloc.size // 4
    nnt = V.nnt3d(g)
    dobs = torch.zeros(nnt * nrec, dtype=torch.float32, device="cuda")
    plan.set_model(ctrue[:n], ctrue[n:2 * n], ctrue[2 * n:])
    plan.model_data(s.souloc, [0], out=dobs.data_ptr(), mem=V.MEM_DEVICE)
    plan.set_model(cstart[:n], cstart[n:2 * n], cstart[2 * n:], padb=padb, randb=randb)
    fg = torch.zeros(1 + 3 * n, dtype=torch.float32, device="cuda")
    stream = torch.cuda.ExternalStream(ctx.stream)

    def step():
        _, mis = plan.gradient(s.souloc, [0], dobs.data_ptr(), V.MEM_DEVICE, fg.data_ptr(),
                               V.MEM_DEVICE)
        if world > 1:
            dist.all_reduce(fg)
        return mis

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = ctx.launches
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # the timed steps run without per-kernel events; the kernel times come
    # from one further step with events on each launch
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            mis = step()
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    launches = ctx.launches - launches0
    ctx.set_timing(True)
    step()
    torch.cuda.synchronize()
    bwd_ms, bwd_n = ctx.kernel_time("bwd3d")
    fwd_ms, fwd_n = ctx.kernel_time("fwd3d")
    ctx.set_timing(False)
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    M = levels(g, flags)
    pts_per_step = 4.0 * (M - 1) * n
    value = pts_per_step * args.steps * world / (ms / 1e3) / 1e9
    # roofline of the dominant kernel (fused backward step)
    upd = (s.nx - 8) * (s.ny - 8) * s.nz
    peak, peak_kind = peaks()
    bwd_avg = bwd_ms / max(bwd_n, 1) / 1e3
    fwd_avg = fwd_ms / max(fwd_n, 1) / 1e3
    achieved = BWD_BYTES_PER_POINT * upd / bwd_avg / 1e9 if bwd_n else None
    # DRAM bytes per updated point from an ncu capture of in-loop launches on
    # a smaller grid (traffic grows with the points updated), scaled to this
    # launch
    traffic = None
    tf = ROOT / "profiles" / "k_bwd3d_tma_traffic.json"
    if tf.exists():
        per_point = json.loads(tf.read_text()).get("dram_bytes_per_point")
        traffic = round(per_point * upd) if per_point else None
    out = None
    if rank == 0:
        e2e = run_e2e(args, ctx, s, cstart, padb, randb, dobs.cpu().numpy(), flags)
        errors = None if args.no_check else oracle_errors(ctx, s, cstart, ctrue, padb, randb,
                                                          CHECK_NT)
        served = None if args.no_served else served_block(args.served_requests, local)
        cpu = None
        if not args.no_cpu:
            import oracle as O
            sh = shortened(s, CPU_SAMPLE_NT)
            d_s = first_samples(dobs.cpu().numpy(), nrec, nnt, V.nnt3d(sh.geom()))
            val, sec = oracle_gradient_sample(sh, cstart, padb, randb, d_s)
            cpu = {"value": round(val, 4), "unit": "Gpts/s", "cores": O.max_threads(),
                   "kind": "port", "sample": cpu_sample_desc(sh, O.max_threads()),
                   "seconds": round(sec, 2)}
        out = {
            "metric": GRADIENT_METRIC,
            "value": round(value, 3), "unit": "Gpts/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded layered VTI model + GRF, Ricker source)",
            "config": gradient_config(args.config, s, M, nrec),
            "misfit": mis,
            "roofline": {"bound": "hbm", "kernel": "k_bwd3d_tma",
                         "achieved": round(achieved, 1) if achieved else None, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": round(achieved / peak, 4) if achieved else None,
                         "traffic": traffic,
                         "bytes_per_point": BWD_BYTES_PER_POINT,
                         "avg_launch_ms": round(bwd_avg * 1e3, 4),
                         "timing": "CUDA events around each launch on the library's stream, "
                                   "one gradient after the timed steps",
                         "fwd3d": {"achieved": round(FWD_BYTES_PER_POINT * upd / fwd_avg / 1e9, 1)
                                   if fwd_n else None,
                                   "avg_launch_ms": round(fwd_avg * 1e3, 4)}},
            "e2e": e2e, "cpu_baseline": cpu, "error_vs_fp64_oracle": errors, "served": served,
            "gpu_launches": launches, "clocks": clk.summary(),
        }
        print(json.dumps(out), flush=True)
    plan.close()
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return out


def run_e2e(args, ctx, s, cstart, padb, randb, dobs, flags):
    """Same metric through the one-call host-buffer C ABI entry point."""
    import torch
    import vtib200 as V
    g = s.geom()
    n = s.nxyz

    def pin(a):
        t = torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).pin_memory()
        return t

    h_cij, h_padb, h_randb, h_dobs = pin(cstart), pin(padb), pin(randb), pin(dobs)
    h_w, h_so, h_rec = pin(s.wavelet), pin(s.souloc), pin(s.recloc)
    h_fg = torch.zeros(1 + 3 * n, dtype=torch.float32).pin_memory()
    shot = np.zeros(1, dtype=np.int32)
    lib = V.lib()
    import ctypes as C
    mis = C.c_double(0)
    nrec = s.recloc.size // 4

    def call():
        ctx.check(lib.vti3d_gradient_cij(
            ctx.handle, C.byref(g), C.c_void_p(h_cij.data_ptr()), C.c_void_p(h_padb.data_ptr()),
            C.c_void_p(h_randb.data_ptr()), C.c_void_p(h_w.data_ptr()),
            C.c_void_p(h_so.data_ptr()), C.c_void_p(shot.ctypes.data), 1,
            C.c_void_p(h_rec.data_ptr()), nrec, C.c_void_p(h_dobs.data_ptr()),
            C.c_void_p(h_fg.data_ptr()), C.byref(mis), flags))

    call()  # warm-up
    steps = max(1, min(args.steps, 2))
    stream = torch.cuda.ExternalStream(ctx.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    t0 = time.perf_counter()
    for _ in range(steps):
        call()
    e1.record(stream)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    ms = max(e0.elapsed_time(e1), wall * 1e3)
    M = levels(g, flags)
    val = 4.0 * (M - 1) * n * steps / (ms / 1e3) / 1e9
    bi = 4 * (cstart.size + padb.size + randb.size + dobs.size + s.wavelet.size)
    return {"value": round(val, 3), "unit": "Gpts/s", "h2d_bytes_per_step": int(bi),
            "d2h_bytes_per_step": int(4 * (1 + 3 * n)), "steps": steps,
            "ms_per_step": round(ms / steps, 2),
            "api": "vti3d_gradient_cij (host buffers; the context keeps the plan "
                   "between calls of the same geometry)"}


def run_parity(args):
    """The full-grid comparison against the FP64 oracle over --nt time samples
    (default: the whole 3000): one GPU gradient, the oracle's FP64 and FP32
    gradients on the host cores; prints one JSON line."""
    import vtib200 as V
    nt = args.nt or CONFIGS[args.config]["nt"]
    s, cstart, ctrue, padb, randb = make_inputs(args.config, 0)
    ctx = V.Context(0)
    try:
        res = oracle_errors(ctx, s, cstart, ctrue, padb, randb, nt)
    finally:
        ctx.close()
    import oracle as O
    res["threads"] = O.max_threads()
    print(json.dumps({"workload": "parity", "config": args.config, **res}), flush=True)
    return res


def run_batched(args):
    """Batched multi-shot gradient (the batching workload): `--shots` shots on
    the 400x400x200 model, each on its own window with apertures per side drawn
    from U{160..400} (seed 5), receivers every 25 m inside each window, all
    shots in one vti3d_batch_gradient call under the schedule
    vti3d_batch_autotune times faster (side by side: one launch per level
    over all windows, CUDA-graph time loops, autotuned segment lengths; per
    shot: each window through the single-grid passes in turn); the other
    schedule is timed once beside it. Compared with the plain per-shot loop on
    the same GPU: vti3d_plan_gradient of one shot at a time on the full model.
    Observed traces are zero (the residual is the modeled data); the work per
    step does not depend on the data values."""
    import torch
    import vtib200 as V
    import vtib200.synth as S

    kw = dict(CONFIGS["gradient400"])
    if args.nt:
        kw["nt"] = args.nt
    s = S.survey3d(**kw)
    wins = S.batch_windows(s.nx, s.ny, args.shots, 160, 400, seed=5)
    souloc, recloc = S.batch_survey3d(s, wins, rec_step=2, rec_depth=25.0, src_depth=25.0)
    g = s.geom()
    n = s.nxyz
    nrec = recloc.size // 4
    nnt = V.nnt3d(g)
    flags = V.OPT_FULL_STEPS
    M = levels(g, flags)
    cs = s.cij()
    torch.cuda.set_device(0)
    ctx = V.Context(0)
    stream = torch.cuda.ExternalStream(ctx.stream)
    b = V.Batch3d(ctx, g, flags)
    b.set_model(cs[:n], cs[n:2 * n], cs[2 * n:])
    b.set_wavelet(s.wavelet)
    b.set_receivers(recloc)
    b.set_shots(souloc, wins, seed=4)
    b.set_schedule({"auto": V.BATCH_AUTO, "side": V.BATCH_SIDE_BY_SIDE,
                    "per_shot": V.BATCH_PER_SHOT}[args.schedule])
    seg_f, seg_b = b.autotune()  # segment lengths, then (auto) the faster schedule
    schedule = b.schedule
    sched_name = {V.BATCH_SIDE_BY_SIDE: "side_by_side", V.BATCH_PER_SHOT: "per_shot"}
    dobs = torch.zeros(nnt * nrec, dtype=torch.float32, device="cuda")
    fg = torch.zeros(1 + 3 * n, dtype=torch.float32, device="cuda")

    def grad(host=None):
        if host is None:
            return b.gradient(dobs.data_ptr(), V.MEM_DEVICE, fg.data_ptr(), V.MEM_DEVICE)[1]
        return b.gradient(host[0], V.MEM_HOST, host[1], V.MEM_HOST)[1]

    # warm-up with direct launches: per-launch device times of the batched kernels
    b.set_options(use_graph=False, seg_fwd=seg_f, seg_bwd=seg_b)
    ctx.set_timing(True)
    grad()
    bwd_ms, bwd_n = ctx.kernel_time("bwd3d")
    fwd_ms, fwd_n = ctx.kernel_time("fwd3d")
    ctx.set_timing(False)
    b.set_options(use_graph=True, seg_fwd=seg_f, seg_bwd=seg_b)
    torch.cuda.synchronize()
    launches0 = ctx.launches
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(0) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            mis = grad()
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    launches = (ctx.launches - launches0) // args.steps
    # the schedule autotune did not choose, one gradient, for the record
    other = V.BATCH_PER_SHOT if schedule == V.BATCH_SIDE_BY_SIDE else V.BATCH_SIDE_BY_SIDE
    other_ms = None
    if args.steps > 0 and not args.no_check:
        b.set_schedule(other)
        grad()
        torch.cuda.synchronize()
        e0.record(stream)
        grad()
        e1.record(stream)
        torch.cuda.synchronize()
        other_ms = e0.elapsed_time(e1)
        b.set_schedule(schedule)
    # end to end: pinned host traces in, host gradient out
    h_dobs = torch.zeros(nnt * nrec, dtype=torch.float32).pin_memory()
    h_fg = torch.zeros(1 + 3 * n, dtype=torch.float32).pin_memory()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    grad((h_dobs.numpy(), h_fg.numpy()))
    e2e_ms = (time.perf_counter() - t0) * 1e3
    area = sum(w[2] * w[3] for w in wins)
    pts = 4.0 * (M - 1) * area * s.nz
    upd = sum((w[2] - 8) * (w[3] - 8) for w in wins) * s.nz
    # windowed plain: the same windows (the batch's own window models and
    # random boundaries), one shot at a time through vti3d_plan_gradient; a
    # sample of the windows is timed and the total scaled by window area
    nwin = max(1, min(args.plain_shots, args.shots))
    pick = sorted(set(int(round(i * (args.shots - 1) / max(nwin - 1, 1))) for i in range(nwin)))
    win_ms, win_area = 0.0, 0
    for j in pick:
        x0, y0, wx, wy = wins[j]
        gs = V.geom3d(wx, wy, g.nz, g.nt, g.npad, g.dx, g.dy, g.dz, g.dt, g.sampling_rate,
                      ox=g.ox + x0 * g.dx, oy=g.oy + y0 * g.dy, oz=g.oz, ot=g.ot)
        ns = wx * wy * g.nz
        cpad, crand = b.shot_models(j)
        randb = np.concatenate([V.get_boundary(crand[k * ns:(k + 1) * ns], wx, wy, g.nz, g.npad)
                                for k in range(3)])
        pw = V.Plan3d(ctx, gs, flags)
        pw.set_model(cpad[:ns], cpad[ns:2 * ns], cpad[2 * ns:], randb=randb)
        pw.set_wavelet(s.wavelet)
        pw.set_receivers(recloc)
        fgw = torch.zeros(1 + 3 * ns, dtype=torch.float32, device="cuda")
        so = souloc[5 * j:5 * j + 5]
        pw.gradient(so, [0], dobs.data_ptr(), V.MEM_DEVICE, fgw.data_ptr(), V.MEM_DEVICE)
        torch.cuda.synchronize()
        e0.record(stream)
        pw.gradient(so, [0], dobs.data_ptr(), V.MEM_DEVICE, fgw.data_ptr(), V.MEM_DEVICE)
        e1.record(stream)
        torch.cuda.synchronize()
        win_ms += e0.elapsed_time(e1)
        win_area += wx * wy
        pw.close()
        del fgw
    windowed_ms = win_ms * area / win_area  # all windows, one at a time
    b.close()
    # plain per-shot loop on the full model
    padb, randb = S.boundaries3d(s)
    plan = V.Plan3d(ctx, g, flags)
    plan.set_model(cs[:n], cs[n:2 * n], cs[2 * n:], padb=padb, randb=randb)
    plan.set_wavelet(s.wavelet)
    plan.set_receivers(recloc)
    nplain = max(1, min(args.plain_shots, args.shots))
    plan.gradient(souloc[:5], [0], dobs.data_ptr(), V.MEM_DEVICE, fg.data_ptr(), V.MEM_DEVICE)
    torch.cuda.synchronize()
    e0.record(stream)
    for k in range(nplain):
        plan.gradient(souloc[5 * k:5 * k + 5], [0], dobs.data_ptr(), V.MEM_DEVICE,
                      fg.data_ptr(), V.MEM_DEVICE)
    e1.record(stream)
    torch.cuda.synchronize()
    plain_ms = e0.elapsed_time(e1) / nplain
    plan.close()
    ctx.close()
    peak, peak_kind = peaks()
    bwd_avg = bwd_ms / max(bwd_n, 1) / 1e3
    fwd_avg = fwd_ms / max(fwd_n, 1) / 1e3
    # bytes over the summed device time of all step launches of one gradient:
    # side by side, every launch covers all windows; per shot, one window
    achieved = (BWD_BYTES_PER_POINT * upd * (M - 1) / (bwd_ms / 1e3) / 1e9
                if bwd_n else None)
    fwd_achieved = (FWD_BYTES_PER_POINT * 2 * upd * (M - 1) / (fwd_ms / 1e3) / 1e9
                    if fwd_n else None)
    shots_s = args.shots / (ms / 1e3)
    plain_s = 1.0 / (plain_ms / 1e3)
    out = {
        "metric": "batched 3D VTI gradient throughput (shots/s), shots on their own windows",
        "value": round(shots_s, 4), "unit": "shots/s", "n_gpus": 1, "steps": args.steps,
        "warmup": 1, "ms_per_step": round(ms, 1), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded layered VTI model + GRF; zero observed traces)",
        "config": {"workload": f"{args.shots} shots, 400x400x200 model, windows U{{160..400}} "
                               f"per side (seed 5), nt={s.nt}, {M} levels, {nrec} receivers",
                   "windows": wins, "segments": [seg_f, seg_b],
                   "graph": schedule == V.BATCH_SIDE_BY_SIDE,
                   "schedule": sched_name[schedule], "misfit": mis},
        "schedules": {sched_name[schedule]: round(ms, 1),
                      sched_name[other]: round(other_ms, 1) if other_ms else None,
                      "unit": "ms per gradient of all shots",
                      "chosen_by": ("vti3d_batch_autotune (one level of each, timed)"
                                    if args.schedule == "auto" else "--schedule")},
        "gpts": round(pts / (ms / 1e3) / 1e9, 2),
        "plain": {"value": round(plain_s, 4), "unit": "shots/s",
                  "ms_per_shot": round(plain_ms, 1), "shots_timed": nplain,
                  "gpts": round(4.0 * (M - 1) * n / (plain_ms / 1e3) / 1e9, 2),
                  "api": "vti3d_plan_gradient, full model, one shot at a time"},
        "speedup_vs_plain": round(shots_s / plain_s, 3),
        "windowed_plain": {"value": round(args.shots / (windowed_ms / 1e3), 4), "unit": "shots/s",
                           "windows_timed": len(pick), "timed_ms": round(win_ms, 1),
                           "api": "vti3d_plan_gradient on each shot's own window (the batch's "
                                  "window models), one at a time; total scaled from the timed "
                                  "windows by window area"},
        "speedup_vs_windowed_plain": round(shots_s / (args.shots / (windowed_ms / 1e3)), 3),
        "roofline": {"bound": "hbm",
                     "kernel": ("k_bwd3d_batch" if schedule == V.BATCH_SIDE_BY_SIDE
                                else "k_bwd3d_tma (one window per launch)"),
                     "achieved": round(achieved, 1) if achieved else None, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": round(achieved / peak, 4) if achieved else None,
                     "traffic": None, "bytes_per_point": BWD_BYTES_PER_POINT,
                     "avg_launch_ms": round(bwd_avg * 1e3, 4), "launches": bwd_n,
                     "fwd3d": {"achieved": round(fwd_achieved, 1) if fwd_achieved else None,
                               "avg_launch_ms": round(fwd_avg * 1e3, 4), "launches": fwd_n}},
        "e2e": {"value": round(args.shots / (e2e_ms / 1e3), 4), "unit": "shots/s",
                "h2d_bytes_per_step": int(4 * nnt * nrec), "d2h_bytes_per_step": int(4 * (1 + 3 * n)),
                "ms_per_step": round(e2e_ms, 1), "api": "vti3d_batch_gradient (host buffers)"},
        "gpu_launches": launches, "clocks": clk.summary(),
    }
    print(json.dumps(out), flush=True)
    return out


def serve_requests(n, budget, chunk, policy, log=None, fwi=None, with_requests=True,
                   device=0):
    """The served form: `n` seeded requests (Poisson 20/s, seed 7) through the
    continuous-batching server; returns its statistics."""
    import vtib200.serve as SV
    srv = SV.Server(device=device, max_bytes=budget, chunk=chunk, keep_results=False, log=log,
                    policy=policy)
    t0 = time.perf_counter()
    st = srv.run(SV.make_requests(n, rate=20.0, seed=7) if with_requests else [], fwi=fwi)
    st["wall_s"] = time.perf_counter() - t0
    st["launches"] = srv.ctx3.launches + srv.ctx2.launches
    srv.close()
    return st


def plain_requests_run(n, log=None, device=0):
    """The plain form of the same requests: one at a time in arrival order on
    one stream (3D through vti3d_plan_*, 2D the same calls)."""
    import vtib200 as V
    import vtib200.serve as SV
    ctx = V.Context(device)
    reqs_p = SV.make_requests(n, rate=20.0, seed=7)
    t0 = time.perf_counter()
    lat = []
    for r in reqs_p:
        now = time.perf_counter() - t0
        if r.arrival > now:
            time.sleep(r.arrival - now)
        if r.dim == 2:
            r.make()(ctx)
        else:
            job = r.make()
            if job.kind == V.JOB_MODEL:
                jc11, jc13, jc33, jw, jso, jrec = job._keep[:6]
                p = V.Plan3d(ctx, job.g, V.OPT_FULL_STEPS)
                p.set_model(jc11, jc13, jc33)
                p.set_wavelet(jw)
                p.set_receivers(jrec)
                p.model_data(jso, [0])
                p.close()
            else:
                SV.plain_gradient(ctx, job)
        lat.append(time.perf_counter() - t0 - r.arrival)
        if log:
            log(f"plain request {r.rid} done at {time.perf_counter() - t0:.2f} s")
    span = time.perf_counter() - t0 - min(r.arrival for r in reqs_p)
    launches = ctx.launches
    ctx.close()
    return {"requests_per_s": round(len(lat) / span, 4), "makespan_s": span,
            "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "launches": launches}


def served_block(n, device=0):
    """The served half of the headline metric, for the default bench line:
    `n` requests served (continuous batching, shortest-first) and the same
    requests one at a time (plain), each request a shot (modeling or
    gradient) of its own grid."""
    served = serve_requests(n, 100 << 30, 32, "sjf", device=device)
    plain = plain_requests_run(n, device=device)
    return {"requests": n,
            "workload": f"{n} requests, Poisson 20/s (seed 7): half 2D 201x401..401x801, half "
                        "3D 128^3..200x400x400, half modeling / half gradient, nt U{2000..4000}, "
                        "Ricker U[10,15] Hz",
            "shots_per_s": round(served["requests_per_s"], 4),
            "p50_s": round(served["p50_s"], 3), "p99_s": round(served["p99_s"], 3),
            "plain_shots_per_s": plain["requests_per_s"],
            "plain_p50_s": round(plain["p50_s"], 3), "plain_p99_s": round(plain["p99_s"], 3),
            "ratio_vs_plain": round(served["requests_per_s"] / plain["requests_per_s"], 3),
            "wall_s": round(served["wall_s"] + plain["makespan_s"], 1)}


def run_served(args):
    """Served workload: Poisson arrivals (mean 20 req/s, seed 7) of mixed
    modeling and gradient requests, half 2D (201x401 .. 401x801) and half 3D
    (128^3 .. 200x400x400), nt U{2000..4000}, Ricker U[10, 15] Hz, random-
    boundary mode, served by the continuous-batching engine (3D) and a second
    stream (2D), with L-BFGS FWI iterations (gradients of shots on windows of
    the 400x400x200 model) interleaved. The plain form serves the same
    requests one at a time in arrival order (3D through vti3d_plan_*, 2D the
    same calls, one stream) and runs the same FWI iterations with
    vti3d_plan_gradient one shot at a time."""
    import torch
    import vtib200 as V
    import vtib200.serve as SV
    import vtib200.synth as S

    torch.cuda.set_device(0)

    def fwi_case():
        kw = dict(CONFIGS["gradient400"])
        kw["nt"] = args.fwi_nt
        s = S.survey3d(**kw)
        tv, te, td = s.extra["true"]
        ctrue = s.cij(tv, te, td)
        g = s.geom()
        wins = S.batch_windows(s.nx, s.ny, args.fwi_shots, 160, 400, seed=5)
        souloc, recloc = S.batch_survey3d(s, wins, rec_step=2, rec_depth=25.0, src_depth=25.0)
        ctx = V.Context(0)
        shots = []
        for k, (x0, y0, wx, wy) in enumerate(wins):
            so = souloc[5 * k:5 * k + 5].copy()
            nr, first = int(so[3]), int(so[4])
            rec = recloc[4 * first:4 * (first + nr)].copy()
            so[4] = 0
            sub = V.geom3d(wx, wy, g.nz, g.nt, g.npad, g.dx, g.dy, g.dz, g.dt, g.sampling_rate,
                           ox=g.ox + x0 * g.dx, oy=g.oy + y0 * g.dy, oz=g.oz)
            p = V.Plan3d(ctx, sub, V.OPT_FULL_STEPS)
            ct = ctrue.reshape(3, g.nz, g.ny, g.nx)[:, :, y0:y0 + wy, x0:x0 + wx]
            p.set_model(*[c.reshape(-1) for c in ct])
            p.set_wavelet(s.wavelet)
            p.set_receivers(rec)
            dobs = p.model_data(so, [0])
            p.close()
            shots.append((so, rec, dobs, (x0, y0, wx, wy)))
        ctx.close()
        c0 = s.cij()
        return g, c0, s.wavelet, shots, float(np.abs(c0).max() * 2e-3)

    log = lambda m: print(m, file=sys.stderr, flush=True)  # noqa: E731
    budget = int(args.budget_gib * (1 << 30))

    def serve(fwi=None):
        return serve_requests(args.requests, budget, args.chunk, args.policy, log, fwi=fwi,
                              with_requests=fwi is None or args.requests_with_fwi)

    def plain_requests():
        return plain_requests_run(args.requests, log)

    with ClockSampler(0) as clk:
        served = serve()
    out = {
        "metric": "served VTI requests: requests/s with p50/p99 latency (continuous batching)",
        "value": round(served["requests_per_s"], 4), "unit": "requests/s", "n_gpus": 1,
        "steps": 1, "warmup": 0, "ms_per_step": round(served["wall_s"] * 1e3, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded requests: layered VTI models, Ricker sources; zero observed "
                "traces for request gradients, modeled traces for the FWI)",
        "config": {"workload": f"{args.requests} requests, Poisson 20/s (seed 7), 2D 201x401.."
                               "401x801 / 3D 128^3..200x400x400, nt U{2000..4000}, Ricker "
                               f"U[10,15] Hz; FWI {args.fwi_iters} iterations x "
                               f"{args.fwi_shots} shots on 400x400x200 windows, nt={args.fwi_nt}",
                   "engine_budget_gib": args.budget_gib, "chunk_ticks": args.chunk,
                   "policy": args.policy},
        "latency_s": {"p50": served["p50_s"], "p99": served["p99_s"]},
        "served": served,
        "gpu_launches": int(served["launches"]), "clocks": clk.summary(),
    }
    if args.plain:
        pl = plain_requests()
        out["plain"] = pl
        out["speedup_vs_plain"] = round(served["requests_per_s"] / pl["requests_per_s"], 3)
    if args.fwi_iters > 0:
        g, c0, w, shots, step0 = fwi_case()
        fwi = SV.FwiDriver(g, c0, w, shots, iterations=args.fwi_iters, step0=step0)
        t0 = time.perf_counter()
        st = serve(fwi)
        out["fwi"] = {"misfits": fwi.misfits, "evaluations": st["fwi_requests"],
                      "wall_s": time.perf_counter() - t0,
                      "requests_beside": st["requests"], "p50_s": st["p50_s"],
                      "p99_s": st["p99_s"]}
        if args.plain:
            ctx = V.Context(0)
            pf = SV.FwiDriver(g, c0, w, shots, iterations=args.fwi_iters, step0=step0)
            t0 = time.perf_counter()
            out["fwi"]["plain_misfits"] = pf.run_plain(ctx)
            out["fwi"]["plain_wall_s"] = time.perf_counter() - t0
            ctx.close()
            out["fwi"]["same_as_plain"] = out["fwi"]["plain_misfits"] == fwi.misfits
    print(json.dumps(out), flush=True)
    return out


def run_gnhv(args):
    """Exact-mode 3D Gauss-Newton H*v plus gradient of one shot (the mixed-
    precision workload): 300 x 600 x 600 at 10 m, nt = 4000 with dt = 0.75 ms
    (1 ms violates the CFL bound for v = 4500 m/s, eps = 0.2, delta = 0.1),
    layered VTI model + Gaussian random field, 12 Hz Ricker, receivers every
    4 cells at 20 m, input vector a seeded Gaussian random field (seed 6) of
    1 % of the model; background checkpoints every K levels in FP32, the
    levels the imaging reads stored as BF16 with per-z-plane FP32 scales,
    misfit in FP64. The error against the FP64 oracle is measured on a
    reduced grid of the same construction (the oracle keeps every level in
    host memory)."""
    import torch
    import vtib200 as V
    import vtib200.synth as S
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O

    torch.cuda.set_device(0)
    nx, ny, nz = args.gn_grid
    nt = args.nt or 4000

    def case(nx, ny, nz, nt, npad):
        s = S.survey3d(nx=nx, ny=ny, nz=nz, nt=nt, npad=npad, d=10.0, dt=7.5e-4, rate=4e-3,
                       freq=12.0, rec_step=4, rec_start=npad, rec_depth=20.0, src_depth=20.0,
                       corr=200.0, smooth_m=None)
        n = s.nxyz
        c = s.cij()
        dc = (S.grf((nz, ny, nx), 200.0 / 10.0, 1.0, 4.0, 6).reshape(-1) * c.reshape(3, -1)
              * 1e-2).reshape(-1).astype(np.float32)
        # observed data: the model with a 2 % smooth velocity perturbation
        vt = s.v * (1 + S.grf((nz, ny, nx), 20.0, 0.02, 0.04, 8).reshape(-1))
        ct = s.cij(vt, s.eps, s.dl)
        return s, c, ct, dc

    bf16 = args.gn_mode == "bf16"
    gflags = V.GNHV_BF16 if bf16 else 0
    # FP32 background: the whole segment of K+1 levels is FP32, so K is chosen
    # near sqrt(2 M) (segment and checkpoint memory balanced)
    gk = args.gn_k if (bf16 or args.gn_k != 126) else max(16, int(round(np.sqrt(2.0 * (nt - 1)))))
    ctx = V.Context(0)
    s, c, ct, dc = case(nx, ny, nz, nt, 40)
    g = s.geom()
    n = s.nxyz
    so = s.souloc[:5].copy()
    so[3], so[4] = s.recloc.size // 4, 0
    cs = [c[k * n:(k + 1) * n] for k in range(3)]
    log = lambda m: print(m, file=sys.stderr, flush=True)  # noqa: E731
    log("model ready")
    dobs = V.gnhv_exact(ctx, g, *[ct[k * n:(k + 1) * n] for k in range(3)], s.wavelet, so,
                        s.recloc, checkpoint_every=gk, want=("traces",))["traces"]
    log("observed traces ready")
    launches0 = ctx.launches
    ctx.set_timing(True)
    with ClockSampler(0) as clk:
        t0 = time.perf_counter()
        out = V.gnhv_exact(ctx, g, *cs, s.wavelet, so, s.recloc, dc=dc, dobs=dobs,
                           checkpoint_every=gk, want=("hv", "grad"), flags=gflags)
        wall = time.perf_counter() - t0
    adj_ms, adj_n = ctx.kernel_time("bwd3d")
    fwd_ms, fwd_n = ctx.kernel_time("fwd3d")
    ctx.set_timing(False)
    launches = ctx.launches - launches0
    ctx.close()
    M = nt - 1
    # pair updates per level: background + Born, recomputation, two adjoints
    pts = 5.0 * (M - 1) * n
    upd = (nx - 8) * (ny - 8) * nz
    peak, peak_kind = peaks()
    adj_avg = adj_ms / max(adj_n, 1) / 1e3
    adj_bytes = 80 if bf16 else 84
    achieved = adj_bytes * upd / adj_avg / 1e9 if adj_n else None
    log("reduced grid vs the FP64 oracle")
    r = args.gn_check
    sr, cr, ctr, dcr = case(r[0], r[1], r[2], args.gn_check_nt, 8)
    gr = sr.geom()
    nr_ = sr.nxyz
    sor = sr.souloc[:5].copy()
    sor[3], sor[4] = sr.recloc.size // 4, 0
    csr = [cr[k * nr_:(k + 1) * nr_] for k in range(3)]
    c64 = [a.astype(np.float64) for a in csr]
    ctx = V.Context(0)
    dob = O.exact_forward3d(gr, *[ctr[k * nr_:(k + 1) * nr_].astype(np.float64)
                                  for k in range(3)], sr.wavelet, sor, [0], sr.recloc)
    gpu = V.gnhv_exact(ctx, gr, *csr, sr.wavelet, sor, sr.recloc, dc=dcr,
                       dobs=dob.astype(np.float32), checkpoint_every=16, flags=gflags)
    ctx.close()
    tr = O.exact_forward3d(gr, *c64, sr.wavelet, sor, [0], sr.recloc)
    bo = O.exact_born3d(gr, *c64, sr.wavelet, sor, [0], sr.recloc, dcr)
    grad = O.exact_adjoint3d(gr, *c64, sr.wavelet, sor, [0], sr.recloc, tr - dob)
    hv = O.exact_adjoint3d(gr, *c64, sr.wavelet, sor, [0], sr.recloc, bo)

    def rel(a, b):
        b = np.asarray(b, dtype=np.float64)
        return float(np.linalg.norm(np.asarray(a, dtype=np.float64) - b) / np.linalg.norm(b))

    errs = {"traces": rel(gpu["traces"], tr), "born_traces": rel(gpu["born"], bo),
            "gradient": rel(gpu["grad"], grad), "hv": rel(gpu["hv"], hv),
            "misfit": abs(gpu["misfit"] - 0.5 * float((tr - dob) @ (tr - dob))) /
            (0.5 * float((tr - dob) @ (tr - dob))),
            "grid": list(r), "nt": args.gn_check_nt}
    res = {
        "metric": "3D exact-mode Gauss-Newton H*v + gradient (grid-point updates/s)",
        "value": round(pts / wall / 1e9, 3), "unit": "Gpts/s", "n_gpus": 1, "steps": 1,
        "warmup": 0, "ms_per_step": round(wall * 1e3, 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 (BF16 stored background)" if bf16 else "f32",
        "data": "synthetic (seeded layered VTI + GRF model, GRF input vector)",
        "config": {"workload": f"GN H*v + gradient, {nx}x{ny}x{nz} at 10 m, nt={nt}, dt=0.75 ms, "
                               f"checkpoints every {gk} levels, "
                               f"{'BF16' if bf16 else 'FP32'} background",
                   "grid": [nx, ny, nz], "nt": nt, "receivers": int(s.recloc.size // 4),
                   "checkpoint_every": gk, "background": args.gn_mode, "misfit": out["misfit"],
                   "updates_per_level": "5 (background+Born, recomputation, 2 adjoints)"},
        "roofline": {"bound": "hbm", "kernel": "k_adj3d_b16" if bf16 else "k_adj3d_tma",
                     "achieved": round(achieved, 1) if achieved else None, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": round(achieved / peak, 4) if achieved else None, "traffic": None,
                     "bytes_per_point": adj_bytes, "avg_launch_ms": round(adj_avg * 1e3, 4),
                     "forward_kernels_ms": round(fwd_ms, 1), "forward_launches": int(fwd_n)},
        "error_vs_fp64_oracle": errs,
        "e2e": {"value": round(pts / wall / 1e9, 3), "unit": "Gpts/s",
                "h2d_bytes_per_step": int(4 * (6 * n + dobs.size)),
                "d2h_bytes_per_step": int(4 * 6 * n),
                "api": "vti3d_gnhv_exact (host buffers)"},
        "gpu_launches": int(launches), "clocks": clk.summary(),
    }
    print(json.dumps(res), flush=True)
    return res


def run_forward2d(args):
    """Plain 2D VTI forward modeling (synthetic_f) of one shot: nz = 201 x
    nx = 401 at 10 m plus a 30-cell pad, dt = 1 ms, 2000 steps, five flat
    layers (v 1500-4500 m/s, eps 0-0.2, delta 0-0.1, seeded interfaces) with a
    -10 % Gaussian velocity anomaly, 15 Hz Ricker at (z 20 m, x 2000 m), 401
    receivers at 20 m; the pad's velocity randomised by the reference's
    random-boundary generator (seed 2, pctG 0.9). Timed on the GPU
    (vti2d_synthetic, host buffers in and out) next to the FP32 oracle on the
    host cores (the reference's 2D path has no CPU implementation)."""
    import torch
    import vtib200 as V
    import vtib200.synth as S
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O

    torch.cuda.set_device(0)
    s = S.survey2d(nx=401, nz=201, nt=2000, npad=30, d=10.0, dt=1e-3, rate=2e-3, freq=15.0,
                   src_x=2000.0, src_z=20.0, rec_z=20.0, seed=1)
    nnx, nnz = s.nx + 2 * s.npad, s.nz + 2 * s.npad
    # velocity of the layered model back from c33 = v^2, randomised pad, back to c
    v = np.sqrt(s.c33).astype(np.float32)
    eps = ((s.c11 / s.c33 - 1) / 2).astype(np.float32)
    dl = ((np.square(s.c13 / s.c33) - 1) / 2).astype(np.float32)
    vr = V.random_boundary_ref(v, nnx, nnz, 1, s.npad, 0.9, 2)
    c11, c13, c33 = V.vepsdel_to_cij(vr, eps, dl)
    g = s.geom()
    ctx = V.Context(0)
    for _ in range(args.warmup):
        V.synthetic_f(ctx, g, c11, c13, c33, s.wavelet, s.sloc, s.rloc, s.taper)
    with ClockSampler(0) as clk:
        ctx.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            tr = V.synthetic_f(ctx, g, c11, c13, c33, s.wavelet, s.sloc, s.rloc, s.taper)
        ctx.synchronize()
        wall = (time.perf_counter() - t0) / args.steps
    ctx.set_timing(True)
    launches0 = ctx.launches
    V.synthetic_f(ctx, g, c11, c13, c33, s.wavelet, s.sloc, s.rloc, s.taper)
    step_ms, step_n = ctx.kernel_time("step2d")
    ctx.set_timing(False)
    launches = ctx.launches - launches0
    snap = V.modeling_f(ctx, g, c11, c13, c33, s.wavelet, int(s.sloc[0] + s.sloc[1] * nnx),
                        s.taper)
    # 14 shots of the same grid with disjoint receiver blocks: all shots in one
    # launch (one cluster each) against the per-level path
    sm = S.survey2d(nx=401, nz=201, nt=2000, npad=30, d=10.0, dt=1e-3, rate=2e-3, freq=15.0,
                    src_z=20.0, rec_z=20.0, seed=1, ns=14)
    sl = sm.sloc.reshape(-1, 4).copy()
    nrb = (sm.rloc.size // 2) // len(sl)
    sl[:, 2] = nrb
    sl[:, 3] = np.arange(len(sl)) * nrb
    multi = {"shots": len(sl), "receivers_per_shot": int(nrb)}
    for key, res in (("resident_ms", True), ("per_level_ms", False)):
        ctx.set_2d_resident(res)
        V.synthetic_f(ctx, g, c11, c13, c33, sm.wavelet, sl.reshape(-1), sm.rloc, s.taper)
        ctx.synchronize()
        t0 = time.perf_counter()
        for _ in range(3):
            V.synthetic_f(ctx, g, c11, c13, c33, sm.wavelet, sl.reshape(-1), sm.rloc, s.taper)
        ctx.synchronize()
        multi[key] = round((time.perf_counter() - t0) / 3 * 1e3, 2)
    ctx.set_2d_resident(True)
    multi["gpts_per_s"] = round(len(sl) * (s.nt - 2) * nnx * nnz / (multi["resident_ms"] / 1e3)
                                / 1e9, 2)
    # the 2D adjoint gradient of the same shot (objFuncGradient_f: forward with
    # checkpoints, exact adjoint with imaging), observed data from the shot
    # itself scaled by 0.9 so the residual is not zero
    dobs = (0.9 * tr).astype(np.float32)
    V.objFuncGradient_f(ctx, g, dobs, c11, c13, c33, s.wavelet, s.sloc, s.rloc, s.taper)
    ctx.synchronize()
    l0 = ctx.launches
    t0 = time.perf_counter()
    for _ in range(3):
        V.objFuncGradient_f(ctx, g, dobs, c11, c13, c33, s.wavelet, s.sloc, s.rloc, s.taper)
    ctx.synchronize()
    gms = (time.perf_counter() - t0) / 3 * 1e3
    grad2d = {"ms_per_shot": round(gms, 2), "levels": 2 * (s.nt - 2),
              "us_per_level": round(gms * 1e3 / (2 * (s.nt - 2)), 2),
              "launches_per_shot": (ctx.launches - l0) // 3,
              "api": "vti2d_gradient (host buffers), per-level kernels launched as "
                     "programmatic dependents"}
    ctx.close()
    pts = (s.nt - 2) * nnx * nnz
    # CPU: the FP32 oracle of the same shot, all host threads
    t0 = time.perf_counter()
    o = O.forward2d(g, c11, c13, c33, s.wavelet, s.sloc, s.rloc, s.taper, dtype=np.float32)
    cpu_s = time.perf_counter() - t0
    o64 = O.forward2d(g, c11, c13, c33, s.wavelet, s.sloc, s.rloc, s.taper)
    err = float(np.linalg.norm(tr.astype(np.float64) - o64) / np.linalg.norm(o64))
    upd = (nnx - 8) * (nnz - 8)
    # one launch per shot (shared-memory resident) or one launch per step
    resident = step_n == 1
    avg = step_ms / ((s.nt - 2) if resident else max(step_n, 1)) / 1e3
    peak, peak_kind = peaks()
    res = {
        "metric": "2D VTI forward modeling throughput (grid-point updates/s)",
        "value": round(pts / wall / 1e9, 3), "unit": "Gpts/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(wall * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded layered VTI model, reference random boundary)",
        "config": {"workload": "2D synthetic_f, 401 x 201 + 30-cell pad, nt 2000, dt 1 ms, "
                               "401 receivers, one shot",
                   "grid": [nnx, nnz], "nt": s.nt, "traces_rel_l2_vs_fp64_oracle": err,
                   "final_snapshot_max": float(np.abs(snap[-1]).max())},
        "roofline": {"bound": "hbm",
                     "kernel": "k_synth2d_resident" if resident else "k_step2d",
                     "achieved": round(36 * upd / avg / 1e9, 1) if step_n else None,
                     "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": round(36 * upd / avg / 1e9 / peak, 4) if step_n else None,
                     "traffic": 0 if resident else None, "bytes_per_point": 36,
                     "avg_step_ms": round(avg * 1e3, 5),
                     "note": ("one launch per shot: the wavefields, taper and c13 stay in the "
                              "shared memory of one 16-CTA cluster for all steps, so there "
                              "is no per-step DRAM traffic; the bound is instruction issue "
                              "on the cluster's 16 SMs, not HBM")
                     if resident else "the whole 2D state (11 arrays x 0.48 MB) fits in L2"},
        "cpu_baseline": {"value": round(pts / cpu_s / 1e9, 4), "unit": "Gpts/s",
                         "cores": os.cpu_count(), "kind": "port",
                         "sample": "the same shot (all 2000 steps), FP32 oracle"},
        "e2e": {"value": round(pts / wall / 1e9, 3), "unit": "Gpts/s",
                "h2d_bytes_per_step": int(4 * (4 * nnx * nnz + s.nt)),
                "d2h_bytes_per_step": int(tr.nbytes), "api": "vti2d_synthetic (host buffers)"},
        "gpu_launches": int(launches), "clocks": clk.summary(),
        "multishot": multi, "gradient2d": grad2d,
    }
    print(json.dumps(res), flush=True)
    return res


def run_reference(args):
    """Reference arm: the reference algorithm's CPU implementation on the host
    cores (the FP32 oracle port: the reference's own CPU path needs ISPC and
    TBB, absent here), all host threads. Each step is one bounded sample of
    the same workload: the whole three-pass gradient of the same shot on the
    full grid over the first CPU_SAMPLE_NT time samples. Inputs are built
    with numpy and the oracle only; the B200 library is never loaded."""
    rank = int(os.environ.get("RANK", 0))
    if rank != 0:
        return None
    import oracle as O
    import vtib200.synth as S
    kw = dict(CONFIGS[args.config])
    host = dict(get_boundary=O.get_boundary, put_boundary=O.put_boundary,
                vepsdel_to_cij=O.vepsdel_to_cij)
    s, cstart, ctrue, padb, randb = S.gradient_inputs(kw, 0, **host)
    nrec = s.recloc.size // 4
    M = levels(OracleGeom(s), 1)
    sh = shortened(s, CPU_SAMPLE_NT)
    n = sh.nxyz
    # observed data of the sample: the FP32 oracle's traces of the true model
    dobs = O.model_data3d(OracleGeom(sh), ctrue[:n], ctrue[n:2 * n], ctrue[2 * n:], sh.wavelet,
                          sh.souloc, [0], sh.recloc, dtype=np.float32, full_steps=True)
    dobs = np.asarray(dobs, dtype=np.float32)
    for _ in range(args.warmup):
        oracle_gradient_sample(sh, cstart, padb, randb, dobs)
    secs = []
    for _ in range(args.steps):
        secs.append(oracle_gradient_sample(sh, cstart, padb, randb, dobs)[1])
    sec = sum(secs)
    pts = 4.0 * (sh.nt - 2) * n * args.steps
    val = pts / sec / 1e9
    thr = O.max_threads()
    import vtib200
    assert vtib200._lib is None, "the reference arm must not load the B200 library"
    out = {"metric": GRADIENT_METRIC,
           "value": round(val, 4), "unit": "Gpts/s", "n_gpus": int(os.environ.get(
               "WORLD_SIZE", 1)), "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": round(sec / args.steps * 1e3, 2), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic (seeded layered VTI model + GRF, Ricker source)",
           "impl": "reference",
           "config": gradient_config(args.config, s, M, nrec),
           "cpu_baseline": {"value": round(val, 4), "unit": "Gpts/s", "cores": thr,
                            "kind": "port",
                            "sample": "each step: " + cpu_sample_desc(sh, thr)},
           "e2e": {"value": round(val, 4), "unit": "Gpts/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--config", default="gradient400", choices=sorted(CONFIGS))
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-check", action="store_true",
                    help="skip the full-grid check against the FP64 oracle")
    ap.add_argument("--no-served", action="store_true",
                    help="skip the served-vs-plain block of the gradient line")
    ap.add_argument("--served-requests", type=int, default=40,
                    help="gradient line: requests of the served-vs-plain block")
    ap.add_argument("--workload", default="gradient",
                    choices=["gradient", "batched", "served", "gnhv", "forward2d", "parity"],
                    help="batched: many shots on their own windows vs the plain loop")
    ap.add_argument("--shots", type=int, default=64, help="batched workload: shots")
    ap.add_argument("--schedule", default="auto", choices=["auto", "side", "per_shot"],
                    help="batched workload: schedule (auto: the one autotune times faster)")
    ap.add_argument("--plain-shots", type=int, default=3,
                    help="batched workload: shots timed in the plain per-shot loop")
    ap.add_argument("--nt", type=int, default=0,
                    help="batched / parity workloads: time samples")
    ap.add_argument("--requests", type=int, default=40, help="served workload: requests")
    ap.add_argument("--budget-gib", type=float, default=100.0,
                    help="served workload: engine device-memory budget (GiB)")
    ap.add_argument("--fwi-iters", type=int, default=10, help="served workload: FWI iterations")
    ap.add_argument("--fwi-shots", type=int, default=20, help="served workload: FWI shots")
    ap.add_argument("--fwi-nt", type=int, default=1000, help="served workload: FWI time samples")
    ap.add_argument("--plain", action="store_true", help="served workload: also the plain form")
    ap.add_argument("--chunk", type=int, default=32, help="served workload: ticks per step")
    ap.add_argument("--policy", default="sjf", choices=["sjf", "fifo"],
                    help="served workload: admission policy of the engine")
    ap.add_argument("--requests-with-fwi", action="store_true",
                    help="served workload: run the requests again beside the FWI")
    ap.add_argument("--gn-grid", type=int, nargs=3, default=[600, 600, 300],
                    help="gnhv workload: nx ny nz")
    ap.add_argument("--gn-k", type=int, default=126, help="gnhv workload: checkpoint interval")
    ap.add_argument("--gn-mode", default="fp32", choices=["bf16", "fp32"],
                    help="gnhv workload: storage of the recomputed background levels (fp32 "
                         "meets the 1e-4 error budget; bf16 halves the segment memory)")
    ap.add_argument("--gn-check", type=int, nargs=3, default=[44, 56, 40],
                    help="gnhv workload: reduced grid of the FP64 oracle check")
    ap.add_argument("--gn-check-nt", type=int, default=300)
    args = ap.parse_args()
    if args.workload == "gnhv" and args.impl == "b200":
        run_gnhv(args)
    elif args.workload == "forward2d" and args.impl == "b200":
        run_forward2d(args)
    elif args.workload == "batched" and args.impl == "b200":
        run_batched(args)
    elif args.workload == "served" and args.impl == "b200":
        run_served(args)
    elif args.workload == "parity" and args.impl == "b200":
        run_parity(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
