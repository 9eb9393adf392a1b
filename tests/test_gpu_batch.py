"""GPU tests of the batched multi-shot 3D gradient (vti3d_batch_*), through
the C ABI.

Every shot of a batch runs on its own window of the model; per shot the
arithmetic is that of vti3d_plan_gradient on a plan whose grid is the window
(objFuncGradientCij3d_f, lib/vti-fwi-3d/gpu/objFuncGradient3d_f.cu:361-1111),
with the window's random boundary generated on the device. The batched result
is checked against per-shot plans given the same window models, and one shot
against the FP64 oracle.
"""
import numpy as np
import pytest

import oracle as O
from conftest import rel_l2

import vtib200 as V
import vtib200.synth as S

pytestmark = pytest.mark.gpu

GRAD_TOL = 1e-4


def _sub_geom(g, win):
    x0, y0, nx, ny = win
    return V.geom3d(nx, ny, g.nz, g.nt, g.npad, g.dx, g.dy, g.dz, g.dt, g.sampling_rate,
                    ox=g.ox + x0 * g.dx, oy=g.oy + y0 * g.dy, oz=g.oz, ot=g.ot)


def _window(a, g, win):
    x0, y0, nx, ny = win
    return a.reshape(g.nz, g.ny, g.nx)[:, y0:y0 + ny, x0:x0 + nx].reshape(-1)


def _split(a, n):
    return [a[k * n:(k + 1) * n] for k in range(3)]


@pytest.fixture(scope="module")
def survey():
    s = S.small3d(nx=100, ny=92, nz=40, nt=150, npad=8, rate=2.1e-3)
    true = S.small3d(nx=100, ny=92, nz=40, nt=150, npad=8, seed=11)
    wins = [(0, 0, 56, 48), (30, 22, 64, 60), (44, 44, 56, 48)]
    souloc, recloc = S.batch_survey3d(s, wins, rec_step=3)
    g = s.geom()
    n = s.nxyz
    return dict(s=s, g=g, n=n, wins=wins, souloc=souloc, recloc=recloc, cij=s.cij(),
                ctrue=true.cij())


def _observed(ctx, k):
    """Observed traces of every shot, modeled on its window of the true model."""
    g, n = k["g"], k["n"]
    nrec = k["recloc"].size // 4
    dobs = np.zeros(V.nnt3d(g) * nrec, dtype=np.float32)
    for j, w in enumerate(k["wins"]):
        gs = _sub_geom(g, w)
        p = V.Plan3d(ctx, gs)
        try:
            p.set_model(*[_window(c, g, w) for c in _split(k["ctrue"], n)])
            p.set_wavelet(k["s"].wavelet)
            p.set_receivers(k["recloc"])
            dobs += p.model_data(k["souloc"][5 * j:5 * j + 5], [0], nrec_total=nrec)
        finally:
            p.close()
    return dobs


def _plan_gradient(ctx, k, b, j, dobs):
    """vti3d_plan_gradient of shot j on its window, with the batch's window
    models (pad model, random boundary)."""
    g = k["g"]
    w = k["wins"][j]
    gs = _sub_geom(g, w)
    ns = w[2] * w[3] * g.nz
    cpad, crand = b.shot_models(j)
    randb = np.concatenate([V.get_boundary(c, w[2], w[3], g.nz, g.npad)
                            for c in _split(crand, ns)])
    p = V.Plan3d(ctx, gs)
    try:
        p.set_model(*_split(cpad, ns), randb=randb)
        p.set_wavelet(k["s"].wavelet)
        p.set_receivers(k["recloc"])
        fg, mis = p.gradient(k["souloc"][5 * j:5 * j + 5], [0], dobs)
    finally:
        p.close()
    return fg, mis, cpad, randb


def _stack(k, parts):
    """Full-model gradient from window gradients, each without its npad x/y
    frame unless that frame is the model's edge."""
    g, n = k["g"], k["n"]
    full = np.zeros((3, g.nz, g.ny, g.nx), dtype=np.float64)
    for (x0, y0, nx, ny), fg in zip(k["wins"], parts):
        ns = nx * ny * g.nz
        xl = 0 if x0 == 0 else g.npad
        xh = nx if x0 + nx == g.nx else nx - g.npad
        yl = 0 if y0 == 0 else g.npad
        yh = ny if y0 + ny == g.ny else ny - g.npad
        for c in range(3):
            a = fg[1 + c * ns:1 + (c + 1) * ns].reshape(g.nz, ny, nx)
            full[c, :, y0 + yl:y0 + yh, x0 + xl:x0 + xh] += a[:, yl:yh, xl:xh]
    return full.reshape(3, -1)


def _batch(ctx, k, seed=17):
    b = V.Batch3d(ctx, k["g"])
    b.set_model(*_split(k["cij"], k["n"]))
    b.set_wavelet(k["s"].wavelet)
    b.set_receivers(k["recloc"])
    b.set_shots(k["souloc"], k["wins"], seed=seed)
    return b


def test_batch_matches_per_shot_plans(ctx, survey):
    k = survey
    dobs = _observed(ctx, k)
    assert np.abs(dobs).max() > 0
    b = _batch(ctx, k)
    try:
        fg, mis = b.gradient(dobs)
        ref = [_plan_gradient(ctx, k, b, j, dobs) for j in range(len(k["wins"]))]
    finally:
        b.close()
    full = _stack(k, [r[0] for r in ref])
    mis_ref = sum(r[1] for r in ref)
    assert mis > 0
    assert abs(mis - mis_ref) / mis_ref < 1e-12
    n = k["n"]
    for c in range(3):
        a = fg[1 + c * n:1 + (c + 1) * n]
        assert np.abs(full[c]).max() > 0
        assert rel_l2(a, full[c]) < 1e-6, c


def test_batch_graph_and_segments_give_the_same_gradient(ctx, survey):
    """CUDA-graph replay and any segment length leave the arithmetic of every
    grid point unchanged: the gradient is bitwise the same."""
    k = survey
    dobs = _observed(ctx, k)
    b = _batch(ctx, k)
    try:
        base, m0 = b.gradient(dobs)
        b.set_options(use_graph=True)
        g1, m1 = b.gradient(dobs)
        g2, m2 = b.gradient(dobs)  # replay of the captured graphs
        b.set_options(use_graph=True, seg_fwd=12, seg_bwd=9)
        g3, m3 = b.gradient(dobs)
        sf, sb = b.autotune()
        g4, m4 = b.gradient(dobs)
    finally:
        b.close()
    assert sf >= 0 and sb >= 0
    for g_, m_ in ((g1, m1), (g2, m2), (g3, m3), (g4, m4)):
        np.testing.assert_array_equal(g_, base)
        assert m_ == m0


def test_batch_per_shot_schedule_gives_the_same_gradient(ctx, survey):
    """The per-shot schedule (each window through the single-grid passes, one
    shot after another) computes every shot with the same arithmetic as the
    side-by-side launches; the misfit sums the same per-shot residuals in the
    same order."""
    k = survey
    dobs = _observed(ctx, k)
    b = _batch(ctx, k)
    try:
        # three windows of at most 64 x 60 cells cannot fill the GPU alone
        assert b.schedule == V.BATCH_SIDE_BY_SIDE
        b.set_schedule(V.BATCH_SIDE_BY_SIDE)
        base, m0 = b.gradient(dobs)
        b.set_schedule(V.BATCH_PER_SHOT)
        assert b.schedule == V.BATCH_PER_SHOT
        g1, m1 = b.gradient(dobs)
        g2, m2 = b.gradient(dobs)  # again, from the state the first left
        b.set_schedule(V.BATCH_AUTO)
        b.autotune()
        assert b.schedule in (V.BATCH_SIDE_BY_SIDE, V.BATCH_PER_SHOT)
        g3, m3 = b.gradient(dobs)
        with pytest.raises(V.VtiError):
            b.set_schedule(7)
    finally:
        b.close()
    np.testing.assert_array_equal(g1, g2)
    assert m1 == m2
    assert abs(m1 - m0) / m0 < 1e-12
    assert abs(m3 - m0) / m0 < 1e-12
    n = k["n"]
    for c in range(3):
        a, ref = g1[1 + c * n:1 + (c + 1) * n], base[1 + c * n:1 + (c + 1) * n]
        assert np.abs(ref).max() > 0
        assert rel_l2(a, ref) < 1e-6, (c, np.abs(a - ref).max())
        assert rel_l2(g3[1 + c * n:1 + (c + 1) * n], ref) < 1e-6, c


def test_batch_f16_traces_equal_the_unpacked_traces(ctx, survey):
    """Observed traces of all shots as one VTI_TRACES_F16 block: each shot's
    slice is expanded on the device to exactly the FP32 traces the block
    stands for, under both schedules."""
    k = survey
    dobs = _observed(ctx, k)
    g = k["g"]
    nnt = V.nnt3d(g)
    nr = k["recloc"].size // 4
    block = V.pack_traces_f16(dobs, nnt)
    dq = V.unpack_traces_f16(block, nr, nnt)
    b = _batch(ctx, k)
    try:
        out = {}
        for sched in (V.BATCH_SIDE_BY_SIDE, V.BATCH_PER_SHOT):
            b.set_schedule(sched)
            b.set_trace_format(V.TRACES_F32)
            out[sched, 32] = b.gradient(dq)
            b.set_trace_format(V.TRACES_F16)
            out[sched, 16] = b.gradient(block)
    finally:
        b.close()
    for sched in (V.BATCH_SIDE_BY_SIDE, V.BATCH_PER_SHOT):
        np.testing.assert_array_equal(out[sched, 16][0], out[sched, 32][0])
        assert out[sched, 16][1] == out[sched, 32][1]


def test_batch_shot_matches_fp64_oracle(ctx, survey):
    """One shot of the batch against the FP64 oracle on its window."""
    k = survey
    dobs = _observed(ctx, k)
    j = 1
    w = k["wins"][j]
    souloc = k["souloc"][5 * j:5 * j + 5]
    b = V.Batch3d(ctx, k["g"])
    try:
        b.set_model(*_split(k["cij"], k["n"]))
        b.set_wavelet(k["s"].wavelet)
        b.set_receivers(k["recloc"])
        b.set_shots(souloc, [w], seed=3)
        fg, mis = b.gradient(dobs)
        cpad, crand = b.shot_models(0)
    finally:
        b.close()
    g = k["g"]
    gs = _sub_geom(g, w)
    ns = w[2] * w[3] * g.nz
    padb = np.concatenate([V.get_boundary(c, w[2], w[3], g.nz, g.npad)
                           for c in _split(cpad, ns)])
    randb = np.concatenate([V.get_boundary(c, w[2], w[3], g.nz, g.npad)
                            for c in _split(crand, ns)])
    o = O.gradient3d(gs, cpad, padb, randb, k["s"].wavelet, souloc, [0], k["recloc"], dobs)
    assert abs(mis - o[0]) / o[0] < 1e-5
    full = _stack(dict(k, wins=[w]), [np.asarray(o, dtype=np.float64)])
    n = k["n"]
    for c in range(3):
        a = fg[1 + c * n:1 + (c + 1) * n]
        assert np.abs(full[c]).max() > 0
        assert rel_l2(a, full[c]) < GRAD_TOL, c


def test_batch_random_boundary_only_lowers_velocity(ctx, survey):
    k = survey
    b = _batch(ctx, k)
    try:
        for j, w in enumerate(k["wins"]):
            cpad, crand = b.shot_models(j)
            np.testing.assert_array_equal(cpad, np.concatenate(
                [_window(c, k["g"], w) for c in _split(k["cij"], k["n"])]))
            r = crand / cpad
            assert r.max() <= 1.0 and r.min() >= 0.7 ** 2 - 1e-6
            ns = w[2] * w[3] * k["g"].nz
            inner = V.zero_boundary(np.ones(ns, dtype=np.float32), w[2], w[3], k["g"].nz,
                                    k["g"].npad)
            for c in range(3):
                rc = r[c * ns:(c + 1) * ns]
                assert np.all(rc[inner == 1] == 1.0)
                assert rc[inner == 0].min() < 0.9
    finally:
        b.close()


def test_batch_rejects_window_outside_model(ctx, survey):
    k = survey
    b = V.Batch3d(ctx, k["g"])
    try:
        b.set_wavelet(k["s"].wavelet)
        b.set_receivers(k["recloc"])
        with pytest.raises(V.VtiError):
            b.set_shots(k["souloc"][:5], [(60, 0, 56, 48)])
    finally:
        b.close()
