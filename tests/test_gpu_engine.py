"""GPU tests of the 3D serving engine (vti3d_engine_*): continuous batching of
modeling and gradient jobs of different grids.

Per job the engine's result is that of a plan on the job's grid
(vti3d_plan_model_data / vti3d_plan_gradient with VTI_OPT_FULL_STEPS, i.e.
modelDataCij3d_f / objFuncGradientCij3d_f, lib/vti-fwi-3d/gpu/modelData3d_f.cu:427,
objFuncGradient3d_f.cu:361), whatever else is admitted beside it: each grid
point's arithmetic does not depend on the other jobs of a launch, so a result
is bitwise the same alone and in a mix.
"""
import numpy as np
import pytest

from conftest import rel_l2

import vtib200 as V
import vtib200.synth as S

pytestmark = pytest.mark.gpu

GiB = 1 << 30


def _split(a, n):
    return [a[k * n:(k + 1) * n] for k in range(3)]


def _survey(nx=48, ny=44, nz=40, nt=130, seed=3, **kw):
    return S.small3d(nx=nx, ny=ny, nz=nz, nt=nt, npad=8, rate=2.1e-3, seed=seed, **kw)


def _grad_job(ctx, s, dobs_seed=11, randb=True):
    g = s.geom()
    n = s.nxyz
    true = _survey(s.nx, s.ny, s.nz, s.nt, seed=dobs_seed)
    p = V.Plan3d(ctx, g, V.OPT_FULL_STEPS)
    try:
        p.set_model(*_split(true.cij(), n))
        p.set_wavelet(s.wavelet)
        p.set_receivers(s.recloc)
        dobs = p.model_data(s.souloc, [0])
    finally:
        p.close()
    padb, rb = S.boundaries3d(s)
    job = V.Engine3d.make_job(V.JOB_GRADIENT, g, *_split(s.cij(), n), s.wavelet, s.souloc,
                              s.recloc, dobs=dobs, randb=rb if randb else None, seed=5)
    return job, dobs, rb


def _run_alone(ctx, job):
    e = V.Engine3d(ctx, 8 * GiB)
    try:
        jid = e.submit(job)
        assert jid is not None
        while e.step(64):
            pass
        ctx.synchronize()
        assert e.poll() == [jid]
        return e.result(jid)
    finally:
        e.close()


def test_engine_gradient_matches_plan(ctx):
    s = _survey()
    job, dobs, rb = _grad_job(ctx, s)
    fg, mis = _run_alone(ctx, job)
    p = V.Plan3d(ctx, s.geom(), V.OPT_FULL_STEPS)
    try:
        p.set_model(*_split(s.cij(), s.nxyz), randb=rb)
        p.set_wavelet(s.wavelet)
        p.set_receivers(s.recloc)
        ref, mref = p.gradient(s.souloc, [0], dobs)
    finally:
        p.close()
    assert mis > 0 and abs(mis - mref) / mref < 1e-12
    assert np.abs(ref[1:]).max() > 0
    assert rel_l2(fg[1:], ref[1:]) < 1e-6


def test_engine_model_matches_plan(ctx):
    s = _survey(nx=56, ny=40, nz=36, nt=150)
    g = s.geom()
    n = s.nxyz
    job = V.Engine3d.make_job(V.JOB_MODEL, g, *_split(s.cij(), n), s.wavelet, s.souloc,
                              s.recloc)
    tr, _ = _run_alone(ctx, job)
    p = V.Plan3d(ctx, g, V.OPT_FULL_STEPS)
    try:
        p.set_model(*_split(s.cij(), n))
        p.set_wavelet(s.wavelet)
        p.set_receivers(s.recloc)
        ref = p.model_data(s.souloc, [0])
    finally:
        p.close()
    assert np.abs(ref).max() > 0
    assert rel_l2(tr, ref) < 1e-6


def test_result_same_alone_and_in_mix(ctx):
    """A gradient job gives the same result alone and admitted, mid-flight,
    beside jobs of other grids (a gradient already in its backward pass and a
    modeling job arriving later)."""
    s = _survey()
    job_a, _, _ = _grad_job(ctx, s, randb=False)
    alone, mis_alone = _run_alone(ctx, job_a)
    other = _survey(nx=64, ny=52, nz=32, nt=110, seed=7)
    job_b, _, _ = _grad_job(ctx, other, dobs_seed=9, randb=False)
    third = _survey(nx=40, ny=48, nz=44, nt=170, seed=8)
    job_c = V.Engine3d.make_job(V.JOB_MODEL, third.geom(), *_split(third.cij(), third.nxyz),
                                third.wavelet, third.souloc, third.recloc)
    e = V.Engine3d(ctx, 8 * GiB)
    try:
        ib = e.submit(job_b)
        e.step(130)  # b is in its backward pass now
        ia = e.submit(job_a)
        e.step(17)
        ic = e.submit(job_c)
        done = {}
        while True:
            active = e.step(25)
            ctx.synchronize()
            for j in e.poll():
                done[j] = e.result(j)
            if not active and len(done) == 3:
                break
        assert set(done) == {ia, ib, ic}
        assert e.stats()[1] == 0  # every job released
    finally:
        e.close()
    fg, mis = done[ia]
    assert mis == mis_alone
    np.testing.assert_array_equal(fg, alone)


def test_admission_by_memory_budget(ctx):
    s = _survey()
    job, _, _ = _grad_job(ctx, s, randb=False)
    e = V.Engine3d(ctx, 1)
    try:
        need = e.job_bytes(job)
    finally:
        e.close()
    e = V.Engine3d(ctx, need + need // 2)
    try:
        a = e.submit(job)
        assert a is not None
        assert e.submit(job) is None  # over budget: VTI_ERR_BUSY, nothing allocated
        assert e.stats()[0] == need
        while e.step(64):
            pass
        ctx.synchronize()
        e.result(a)
        assert e.stats()[0] == 0
        b = e.submit(job)  # admitted once the first job has left
        assert b is not None
    finally:
        e.close()
