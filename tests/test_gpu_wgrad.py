"""GPU parity of the source-wavelet gradient, called through the C ABI:
waveletGradientCij3d_f (lib/vti-fwi-3d/gpu/modelData3d_f.cu) and
waveletGradient_f (lib/vti-fwi-2d/objFuncGradient_f.cu) against the FP64
oracle and the reference's own output. A wavelet gradient is a sum of adjoint
samples over levels, held to the gradient tolerance (relative L2 1e-4)."""
import numpy as np
import pytest

import cases as K
import oracle as O
from conftest import load_golden, rel_l2

import vtib200 as V

pytestmark = pytest.mark.gpu

WGRAD_TOL = 1e-4


def _split(cij, n):
    return cij[:n], cij[n:2 * n], cij[2 * n:]


@pytest.mark.parametrize("name", K.WGRAD_CASES3D)
def test_wavelet_gradient3d_matches_oracle_and_reference(ctx, name):
    c = K.case3d(name)
    s = c["s"]
    g = s.geom()
    n = s.nxyz
    model = K.pad_model3d(c)
    dobs = load_golden(name)["dobs"]
    gw = V.waveletGradientCij3d_f(ctx, g, s.souloc, c["shotid"], s.recloc, *_split(model, n),
                                  dobs)
    o = O.wavelet_gradient3d(g, *_split(model, n), s.souloc, c["shotid"], s.recloc, dobs)
    assert np.abs(o).max() > 0
    assert rel_l2(gw, o) < WGRAD_TOL
    assert rel_l2(gw, load_golden(f"{name}_wgrad")["gwavelet"]) < WGRAD_TOL


def test_wavelet_gradient3d_is_linear_in_the_traces(ctx):
    c = K.case3d("g3_b")
    s = c["s"]
    g = s.geom()
    n = s.nxyz
    model = K.pad_model3d(c)
    dobs = load_golden("g3_b")["dobs"]
    a = V.waveletGradientCij3d_f(ctx, g, s.souloc, c["shotid"], s.recloc, *_split(model, n), dobs)
    b = V.waveletGradientCij3d_f(ctx, g, s.souloc, c["shotid"], s.recloc, *_split(model, n),
                                 -3.0 * dobs)
    assert np.abs(a).max() > 0
    assert rel_l2(b, -3.0 * a) < 1e-6


@pytest.mark.parametrize("name", K.WGRAD_CASES2D)
def test_wavelet_gradient2d_matches_oracle_and_reference(ctx, name):
    s = K.case2d(name)["s"]
    g = s.geom()
    dobs = load_golden(name)["dobs"]
    gw = V.waveletGradient_f(ctx, g, dobs, s.c11, s.c13, s.c33, s.sloc, s.rloc, s.taper)
    o = O.wavelet_gradient2d(g, s.c11, s.c13, s.c33, s.sloc, s.rloc, s.taper, dobs)
    assert np.abs(o).max() > 0
    assert rel_l2(gw, o) < WGRAD_TOL
    assert rel_l2(gw, load_golden(f"{name}_wgrad")["gwavelet"]) < WGRAD_TOL
