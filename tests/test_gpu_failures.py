"""Failure paths of the library, exercised without faulting the GPU.

* Unstable time steps: every entry point that takes a model refuses one
  whose leapfrog number dt^2 lambda_max is not below 4 with VTI_ERR_CFL
  before it computes anything (the reference would run it and return growing
  values). The check runs on the device for plans and batches (over the
  uploaded volumes, random boundary included) and on the host for the 2D
  path, the serving engine and the Gauss-Newton product.
* VTI_OPT_CHECK_FINITE: a model holding a NaN in one cell (a stable dt
  otherwise) makes the wavefields non-finite; the call reports
  VTI_ERR_NONFINITE instead of returning NaN gradients silently.
* Bounded waits: a kernel waiting on an mbarrier that nothing completes gives
  up after its poll limit and the host sees VTI_ERR_TIMEOUT through the
  context status word; the context stays usable afterwards.
"""
import ctypes as C

import numpy as np
import pytest

import cases as K

import vtib200 as V
import vtib200.synth as S

pytestmark = pytest.mark.gpu


def _unstable_geom(g, factor=2.0):
    """The same geometry with dt scaled so dt^2 lambda_max >= 4."""
    import copy
    u = copy.copy(g)
    u.dt = g.dt * factor
    u.sampling_rate = g.sampling_rate * factor
    return u


def test_plan_refuses_an_unstable_model(ctx):
    s = S.small3d(nx=40, ny=36, nz=32, nt=60, npad=8)
    n = s.nxyz
    c = s.cij()
    g = s.geom()
    assert V.cfl_number(g, c[:n], c[n:2 * n], c[2 * n:]) < 4
    ug = _unstable_geom(g, 2.5)
    assert V.cfl_number(ug, c[:n], c[n:2 * n], c[2 * n:]) >= 4
    p = V.Plan3d(ctx, ug, V.OPT_FULL_STEPS)
    try:
        with pytest.raises(V.VtiError) as e:
            p.set_model(c[:n], c[n:2 * n], c[2 * n:])
        assert e.value.status == V.VTI_ERR_CFL
        assert "stability bound" in str(e.value)
        # nothing runs on a refused model
        p.set_wavelet(s.wavelet)
        p.set_receivers(s.recloc)
        with pytest.raises(V.VtiError) as e:
            p.model_data(s.souloc, [0])
        assert e.value.status == V.VTI_ERR_ARG
    finally:
        p.close()
    # the one-call form and the drop-in conventions report it as well
    padb, randb = S.boundaries3d(s)
    with pytest.raises(V.VtiError) as e:
        V.objFuncGradientCij3d_f(ctx, ug, s.souloc, [0], s.recloc, s.wavelet, c, padb, randb,
                                 np.zeros(V.nnt3d(ug) * (s.recloc.size // 4), np.float32))
    assert e.value.status == V.VTI_ERR_CFL
    # a stable call on the same context still works
    d = V.modelDataCij3d_f(ctx, g, s.souloc, [0], s.recloc, s.wavelet, c[:n], c[n:2 * n],
                           c[2 * n:], flags=V.OPT_FULL_STEPS)
    assert np.isfinite(d).all() and np.abs(d).max() > 0


def test_2d_entry_points_refuse_an_unstable_model(ctx):
    s = K.case2d("g2_a")["s"]
    g = s.geom()
    assert V.cfl_number2d(g, s.c11, s.c13, s.c33) < 4
    g.dt *= 2.5
    g.rate *= 2.5
    assert V.cfl_number2d(g, s.c11, s.c13, s.c33) >= 4
    for fn in (V.synthetic_f, ):
        with pytest.raises(V.VtiError) as e:
            fn(ctx, g, s.c11, s.c13, s.c33, s.wavelet, s.sloc, s.rloc, s.taper)
        assert e.value.status == V.VTI_ERR_CFL
    rows = (g.nt - 1) // int(np.float32(g.rate) / np.float32(g.dt) + np.float32(0.5)) + 1
    nr = V._i32(s.rloc).size // 2
    data = np.zeros(rows * nr, np.float32)
    with pytest.raises(V.VtiError) as e:
        V.objFuncGradient_f(ctx, g, data, s.c11, s.c13, s.c33, s.wavelet, s.sloc, s.rloc, s.taper)
    assert e.value.status == V.VTI_ERR_CFL


def test_a_nan_model_is_refused(ctx):
    s = S.small3d(nx=40, ny=36, nz=32, nt=60, npad=8)
    c = s.cij()
    padb, randb = S.boundaries3d(s)
    g = s.geom()
    bad = c.copy()
    bad[(20 * s.ny + 18) * s.nx + 20] = np.nan
    dobs = np.zeros(V.nnt3d(g) * (s.recloc.size // 4), np.float32)
    with pytest.raises(V.VtiError) as e:
        V.objFuncGradientCij3d_f(ctx, g, s.souloc, [0], s.recloc, s.wavelet, bad, padb, randb,
                                 dobs)
    assert e.value.status == V.VTI_ERR_CFL


def test_check_finite_reports_non_finite_wavefields(ctx):
    """An infinite source sample makes the wavefield non-finite: with
    VTI_OPT_CHECK_FINITE the scan after the pass reports it; without it the
    call returns the non-finite traces as the reference would."""
    s = S.small3d(nx=40, ny=36, nz=32, nt=60, npad=8)
    n = s.nxyz
    c = s.cij()
    g = s.geom()
    w = s.wavelet.copy()
    w[10] = np.inf
    args = (ctx, g, s.souloc, [0], s.recloc, w, c[:n], c[n:2 * n], c[2 * n:])
    d = V.modelDataCij3d_f(*args, flags=V.OPT_FULL_STEPS)
    assert not np.isfinite(d).all()
    with pytest.raises(V.VtiError) as e:
        V.modelDataCij3d_f(*args, flags=V.OPT_FULL_STEPS | V.OPT_CHECK_FINITE)
    assert e.value.status == V.VTI_ERR_NONFINITE
    # the gradient path: an infinite observed sample poisons the adjoint
    padb, randb = S.boundaries3d(s)
    dobs = np.zeros(V.nnt3d(g) * (s.recloc.size // 4), np.float32)
    dbad = dobs.copy()
    dbad[5] = np.inf
    with pytest.raises(V.VtiError) as e:
        V.objFuncGradientCij3d_f(ctx, g, s.souloc, [0], s.recloc, s.wavelet, c, padb, randb,
                                 dbad, flags=V.OPT_FULL_STEPS | V.OPT_CHECK_FINITE)
    assert e.value.status == V.VTI_ERR_NONFINITE
    # the context is still usable and a clean call passes the scans
    fg, mis = V.objFuncGradientCij3d_f(ctx, g, s.souloc, [0], s.recloc, s.wavelet, c, padb,
                                       randb, dobs, flags=V.OPT_FULL_STEPS | V.OPT_CHECK_FINITE)
    assert np.isfinite(fg).all() and mis > 0


def test_bounded_wait_gives_up_and_reports_a_timeout(ctx):
    st = V.lib().vti_ctx_check_bounded_wait(ctx.handle, C.c_uint(2000))
    assert st == V.VTI_ERR_TIMEOUT
    assert b"timed out" in V.lib().vti_ctx_last_error(ctx.handle)
    assert V.lib().vti_ctx_check_bounded_wait(ctx.handle, C.c_uint(0)) == V.VTI_ERR_ARG
    # the status word was cleared and the context works
    s = S.small3d(nx=40, ny=36, nz=32, nt=60, npad=8)
    n = s.nxyz
    c = s.cij()
    d = V.modelDataCij3d_f(ctx, s.geom(), s.souloc, [0], s.recloc, s.wavelet, c[:n],
                           c[n:2 * n], c[2 * n:], flags=V.OPT_FULL_STEPS)
    assert np.isfinite(d).all() and np.abs(d).max() > 0
