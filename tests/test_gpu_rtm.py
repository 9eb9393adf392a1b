"""GPU parity of reverse-time migration, called through the C ABI:
rtmCij3d_f (lib/vti-fwi-3d/gpu/rtm3d_f.cu) and rtm_f (lib/vti-fwi-2d/rtm_f.cu)
against the FP64 oracle and the reference's own images.

An image sums products of two FP32 wavefields over every level, like a
gradient, so it is held to the gradient tolerance (relative L2 1e-4).
"""
import numpy as np
import pytest

import cases as K
import oracle as O
from conftest import load_golden, rel_l2

import vtib200 as V
import vtib200.synth as S

pytestmark = pytest.mark.gpu

IMAGE_TOL = 1e-4


def _split(cij, n):
    return cij[:n], cij[n:2 * n], cij[2 * n:]


@pytest.mark.parametrize("name", K.RTM_CASES3D)
def test_rtm3d_matches_oracle_and_reference(ctx, name):
    c = K.case3d(name)
    s = c["s"]
    g = s.geom()
    n = s.nxyz
    model = K.rtm_model3d(c)
    dobs = load_golden(name)["dobs"]
    img = V.rtmCij3d_f(ctx, g, s.souloc, c["shotid"], s.recloc, s.wavelet, *_split(model, n),
                       dobs)
    o = O.rtm3d(g, *_split(model, n), s.wavelet, s.souloc, c["shotid"], s.recloc, dobs)
    assert np.abs(o).max() > 0
    assert rel_l2(img, o) < IMAGE_TOL
    assert rel_l2(img, load_golden(f"{name}_rtm")["image"]) < IMAGE_TOL


def test_rtm3d_plan_matches_one_call_and_is_linear_in_data(ctx):
    """A resident plan gives the one-call image bit for bit, twice in a row
    (the image is cleared per call), and the image is linear in the traces."""
    c = K.case3d("g3_b")
    s = c["s"]
    g = s.geom()
    n = s.nxyz
    model = K.rtm_model3d(c)
    dobs = load_golden("g3_b")["dobs"]
    one = V.rtmCij3d_f(ctx, g, s.souloc, c["shotid"], s.recloc, s.wavelet, *_split(model, n), dobs)
    p = V.Plan3d(ctx, g)
    try:
        p.set_model(*_split(model, n))
        p.set_wavelet(s.wavelet)
        p.set_receivers(s.recloc)
        a = p.rtm(s.souloc, c["shotid"], dobs)
        b = p.rtm(s.souloc, c["shotid"], dobs)
        twice = p.rtm(s.souloc, c["shotid"], 2.0 * dobs)
    finally:
        p.close()
    np.testing.assert_array_equal(a, one)
    np.testing.assert_array_equal(b, one)
    assert np.abs(one).max() > 0
    assert rel_l2(twice, 2.0 * one) < 1e-6


@pytest.mark.parametrize("name", K.RTM_CASES2D)
def test_rtm2d_matches_oracle_and_reference(ctx, name):
    s = K.case2d(name)["s"]
    g = s.geom()
    dobs = load_golden(name)["dobs"]
    img = V.rtm_f(ctx, g, dobs, s.c11, s.c13, s.c33, s.wavelet, s.sloc, s.rloc, s.taper)
    o = O.rtm2d(g, s.c11, s.c13, s.c33, s.wavelet, s.sloc, s.rloc, s.taper, dobs)
    assert np.abs(o).max() > 0
    assert rel_l2(img, o) < IMAGE_TOL
    assert rel_l2(img, load_golden(f"{name}_rtm")["image"]) < IMAGE_TOL


def test_rtm2d_every_step_sampled_matches_oracle(ctx):
    """rate == dt: level 1 is a slice of its own and every step is imaged
    against exact slices; three shots share the slice store."""
    s = S.survey2d(nx=56, nz=36, nt=160, npad=8, d=10.0, dt=1e-3, rate=1e-3, freq=20.0,
                   src_x=250.0, src_z=40.0, rec_z=20.0, ns=3)
    g = s.geom()
    data = V.synthetic_f(ctx, g, s.c11, s.c13, s.c33, s.wavelet, s.sloc, s.rloc, s.taper)
    img = V.rtm_f(ctx, g, data, s.c11, s.c13, s.c33, s.wavelet, s.sloc, s.rloc, s.taper)
    o = O.rtm2d(g, s.c11, s.c13, s.c33, s.wavelet, s.sloc, s.rloc, s.taper, data)
    assert np.abs(o).max() > 0
    assert rel_l2(img, o) < IMAGE_TOL


@pytest.mark.parametrize("name", sorted(K.ODCIG_CASES2D))
def test_odcig2d_matches_oracle_and_reference(ctx, name):
    """odcig_f: offset-domain common-image gathers."""
    s = K.case2d(name)["s"]
    g = s.geom()
    nhx = K.ODCIG_CASES2D[name]
    dobs = load_golden(name)["dobs"]
    img = V.odcig_f(ctx, g, nhx, dobs, s.c11, s.c13, s.c33, s.wavelet, s.sloc, s.rloc, s.taper)
    o = O.odcig2d(g, nhx, s.c11, s.c13, s.c33, s.wavelet, s.sloc, s.rloc, s.taper, dobs)
    assert np.abs(o).max() > 0
    assert rel_l2(img, o) < IMAGE_TOL
    ref = load_golden(f"{name}_odcig")["image"].reshape(2 * nhx + 1, -1)
    assert rel_l2(img, ref) < IMAGE_TOL
    # every offset panel carries signal
    assert all(np.abs(ref[h]).max() > 0 for h in range(2 * nhx + 1))


@pytest.mark.parametrize("nlag", [3, 6])
def test_odcig3d_lag0_is_the_rtm_image_and_matches_oracle(ctx, nlag):
    """Offset-domain gathers (odcig3d_f's extended imaging condition): the
    zero-lag gather is the RTM image bit for bit on the imaged x range
    [max(4, nlag), nx - max(4, nlag)) and zero outside it; every lag matches
    the FP64 oracle. nlag = 6 > 4 exercises the narrowed x range."""
    c = K.case3d("g3_a")
    s = c["s"]
    g = s.geom()
    n = s.nxyz
    model = K.rtm_model3d(c)
    dobs = load_golden("g3_a")["dobs"]
    p = V.Plan3d(ctx, g)
    try:
        p.set_model(*_split(model, n))
        p.set_wavelet(s.wavelet)
        p.set_receivers(s.recloc)
        img = p.rtm(s.souloc, c["shotid"], dobs)
        gat = p.odcig(s.souloc, c["shotid"], dobs, nlag)
    finally:
        p.close()
    assert gat.shape == (2 * nlag + 1, n)
    lo = max(4, nlag)
    mask = np.zeros((s.nz, s.ny, s.nx), dtype=bool)
    mask[:, :, lo:s.nx - lo] = True
    mask = mask.reshape(-1)
    np.testing.assert_array_equal(gat[nlag][mask], img[mask])
    assert not gat[:, ~mask].any()
    o = O.odcig3d(g, *_split(model, n), s.wavelet, s.souloc, c["shotid"], s.recloc, dobs, nlag)
    for k in range(2 * nlag + 1):
        assert np.abs(o[k]).max() > 0, k
        assert rel_l2(gat[k], o[k]) < IMAGE_TOL, k
