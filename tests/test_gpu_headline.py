"""Parity on the full grid of the headline gradient workload.

The benchmark's gradient runs on a 400 x 400 x 200 grid (40-cell pad inside)
with the layered VTI + Gaussian-random-field model, a 12 Hz Ricker source at
the centre and a 200 x 200 receiver grid. Here the same grid, model, source
and receivers run with the time axis cut to nt = 130 (129 levels of each
pass) so that the FP64 oracle finishes in seconds of host time; every tile,
z-segment and boundary path of the full-size launches is exercised. The calls
go through the host-buffer C ABI (vti3d_model_data_cij, vti3d_gradient_cij)
with VTI_OPT_FULL_STEPS, as the benchmark runs them.

Tolerances (relative L2 against the FP64 oracle): FP32 traces and misfit
1e-5. Gradients: at this nt the whole gradient norm sits within two cells of
the source point (the imaging sum of the source's Laplacian spike), where the
reference's random-boundary time reversal in FP32 leaves a rounding noise of
2e-5 to 2.2e-4 depending only on the order of the FP32 operations: eight
equivalent evaluation orders of the same algorithm, run through the oracle,
spread over that range (the reference's own, with stencil sums in double,
gives 1.1e-4 for c11). The bar is therefore the top of that envelope with
margin, 3e-4, and the FP32 oracle (the reference algorithm restated in FP32)
must fall inside it too; the GPU and the FP64 oracle agree to 1e-6 on the
traces and the misfit.
"""
import numpy as np
import pytest

import oracle as O
from conftest import rel_l2

import vtib200 as V
import vtib200.synth as S

pytestmark = pytest.mark.gpu

TRACE_TOL = 1e-5
GRAD_TOL = 3e-4  # FP32 rounding envelope of the source-point imaging sum at this nt
NT = 130


@pytest.fixture(scope="module")
def headline():
    s, cstart, ctrue, padb, randb = S.gradient_inputs(dict(S.GRADIENT400, nt=NT))
    return s, cstart, ctrue, padb, randb


def _split(c, n):
    return c[:n], c[n:2 * n], c[2 * n:]


def test_headline_grid_traces_misfit_and_gradient_match_the_oracle(ctx, headline):
    s, cstart, ctrue, padb, randb = headline
    g = s.geom()
    n = s.nxyz
    assert (s.nx, s.ny, s.nz, s.npad) == (400, 400, 200, 40)
    flags = V.OPT_FULL_STEPS
    dobs = V.modelDataCij3d_f(ctx, g, s.souloc, [0], s.recloc, s.wavelet, *_split(ctrue, n),
                              flags=flags)
    dmod = V.modelDataCij3d_f(ctx, g, s.souloc, [0], s.recloc, s.wavelet, *_split(cstart, n),
                              flags=flags)
    fg, mis = V.objFuncGradientCij3d_f(ctx, g, s.souloc, [0], s.recloc, s.wavelet, cstart, padb,
                                       randb, dobs, flags=flags)
    assert np.isfinite(fg).all()
    for dtype in (np.float64, np.float32):
        o, mod = O.gradient3d(g, cstart, padb, randb, s.wavelet, s.souloc, [0], s.recloc, dobs,
                              dtype=dtype, full_steps=True, want_modeled=True)
        assert np.abs(mod).max() > 0 and o[0] > 0
        assert rel_l2(dmod, mod) < TRACE_TOL, dtype
        assert abs(mis - o[0]) / o[0] < TRACE_TOL, dtype
        for k in range(3):
            a, b = fg[1 + k * n:1 + (k + 1) * n], o[1 + k * n:1 + (k + 1) * n]
            assert np.abs(b).max() > 0
            assert rel_l2(a, b) < GRAD_TOL, (dtype, k, rel_l2(a, b))


def test_headline_gradient_is_bitwise_reproducible(ctx, headline):
    """Every launch of the step kernels computes each cell once, from its own
    stage of a TMA ring; the same inputs therefore give the same bits, call
    after call. The time-reversed reconstruction amplifies any read of a
    wrong stage row by orders of magnitude within a few dozen levels, so a
    race between the consumers' shared-memory reads and the ring's refill
    shows here (it did, once per ~1000 backward launches, before the stage
    release carried a proxy fence)."""
    s, cstart, ctrue, padb, randb = headline
    g = s.geom()
    n = s.nxyz
    flags = V.OPT_FULL_STEPS
    p = V.Plan3d(ctx, g, flags)
    try:
        p.set_wavelet(s.wavelet)
        p.set_receivers(s.recloc)
        nr = s.recloc.size // 4
        p.set_model(*_split(ctrue, n), padb=padb, randb=randb)
        dobs = p.model_data(s.souloc, [0], nrec_total=nr)
        p.set_model(*_split(cstart, n), padb=padb, randb=randb)
        runs = [p.gradient(s.souloc, [0], dobs) for _ in range(4)]
        images = [p.rtm(s.souloc, [0], dobs) for _ in range(3)]
    finally:
        p.close()
    for fg, mis in runs[1:]:
        assert mis == runs[0][1]
        np.testing.assert_array_equal(fg, runs[0][0])
    for im in images[1:]:
        np.testing.assert_array_equal(im, images[0])

