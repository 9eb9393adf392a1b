"""CPU tests of the oracle: pinned against the reference's own GPU outputs
(golden fixtures made by tests/golden/make_golden.py from the unmodified
reference sources), plus self-consistency properties."""
import numpy as np
import pytest

import cases as K
import oracle as O
from conftest import load_golden, rel_l2

import vtib200.synth as S


def _split(cij, n):
    return cij[:n], cij[n:2 * n], cij[2 * n:]


@pytest.mark.parametrize("name", K.CASES3D)
def test_oracle_model_data_matches_reference(name):
    c = K.case3d(name)
    s = c["s"]
    gold = load_golden(name)
    assert str(gold["inputs"]) == K.digest(s.souloc, s.recloc, s.wavelet, c["cij"],
                                           c["cij_true"], c["padb"], c["randb"])
    g = s.geom()
    n = s.nxyz
    for key, cij in (("dobs", c["cij_true"]), ("ddata", c["cij"])):
        d = O.model_data3d(g, *_split(cij, n), s.wavelet, s.souloc, c["shotid"], s.recloc)
        assert np.abs(gold[key]).max() > 0
        assert rel_l2(d, gold[key]) < 1e-5, key
        # same recorded / unrecorded samples as the reference's bookkeeping
        # (FP64 leading-edge values the FP32 reference underflows are ignored)
        nnt = O.nnt3d(g)
        thr = 1e-9 * np.abs(gold[key]).max()
        ours = (np.abs(d) > thr).reshape(-1, nnt).any(axis=0)
        theirs = (np.abs(gold[key]) > thr).reshape(-1, nnt).any(axis=0)
        assert np.array_equal(ours, theirs), key


@pytest.mark.parametrize("name", K.GRAD_CASES3D)
def test_oracle_gradient_matches_reference(name):
    c = K.case3d(name)
    s = c["s"]
    gold = load_golden(name)
    g = s.geom()
    fg = O.gradient3d(g, c["cij"], c["padb"], c["randb"], s.wavelet, s.souloc, c["shotid"],
                      s.recloc, gold["dobs"])
    ref = gold["fgcij"].astype(np.float64)
    assert abs(fg[0] - ref[0]) / abs(ref[0]) < 1e-5
    n = s.nxyz
    for k in range(3):
        assert rel_l2(fg[1 + k * n:1 + (k + 1) * n], ref[1 + k * n:1 + (k + 1) * n]) < 1e-4, k


def _digest2d(c):
    s = c["s"]
    return K.digest(s.c11, s.c13, s.c33, s.taper, s.wavelet, s.sloc, s.rloc,
                    *c["true"].values(), *c["dc"].values())


@pytest.mark.parametrize("name", K.CASES2D)
def test_oracle_2d_gradient_and_gn_product_match_reference(name):
    c = K.case2d(name)
    s = c["s"]
    gold = load_golden(name)
    assert str(gold["inputs"]) == _digest2d(c)
    g = s.geom()
    n = (s.nx + 2 * s.npad) * (s.nz + 2 * s.npad)
    g11, g13, g33, mis = O.gradient2d(g, s.c11, s.c13, s.c33, s.wavelet, s.sloc, s.rloc, s.taper,
                                      data=gold["dobs"])
    ref = gold["grad"]
    assert abs(mis - ref[3 * n]) / ref[3 * n] < 1e-5
    for k, a in enumerate((g11, g13, g33)):
        assert np.abs(ref[k * n:(k + 1) * n]).max() > 0
        assert rel_l2(a, ref[k * n:(k + 1) * n]) < 1e-4, k
    h = O.gradient2d(g, s.c11, s.c13, s.c33, s.wavelet, s.sloc, s.rloc, s.taper,
                     dc=(c["dc"]["c11"], c["dc"]["c13"], c["dc"]["c33"]))
    ref = gold["gnhess"]
    for k in range(3):
        assert np.abs(ref[k * n:(k + 1) * n]).max() > 0
        assert rel_l2(h[k], ref[k * n:(k + 1) * n]) < 1e-4, k


@pytest.mark.parametrize("name", K.CASES2D)
def test_oracle_2d_matches_reference(name):
    c = K.case2d(name)
    s = c["s"]
    gold = load_golden(name)
    assert str(gold["inputs"]) == _digest2d(c)
    g = s.geom()
    d = O.forward2d(g, s.c11, s.c13, s.c33, s.wavelet, s.sloc, s.rloc, s.taper)
    assert rel_l2(d.reshape(-1), gold["data"]) < 1e-5
    w = O.forward2d(g, s.c11, s.c13, s.c33, s.wavelet, None, None, s.taper, mode=1,
                    slocxz=int(s.sloc[0] + s.sloc[1] * (s.nx + 2 * s.npad)))
    # whole-wavefield snapshots: the reference's FP32 rounding is ~1e-5 here
    assert rel_l2(w[gold["snap_rows"]], gold["snaps"]) < 2e-5


def test_oracle_fp32_tracks_fp64():
    c = K.case3d("g3_a")
    s = c["s"]
    g = s.geom()
    n = s.nxyz
    d64 = O.model_data3d(g, *_split(c["cij"], n), s.wavelet, s.souloc, c["shotid"], s.recloc)
    d32 = O.model_data3d(g, *_split(c["cij"], n), s.wavelet, s.souloc, c["shotid"], s.recloc,
                         dtype=np.float32)
    assert rel_l2(d32, d64) < 1e-5


def test_oracle_accepts_float64_inputs():
    """Inputs converted to float32 for the call give the float32 result (the
    converted copies must live until the call returns)."""
    c = K.case3d("g3_a")
    s = c["s"]
    g = s.geom()
    dobs = load_golden("g3_a")["dobs"]
    args = (g, c["cij"], c["padb"], c["randb"], s.wavelet, s.souloc, c["shotid"], s.recloc)
    a = O.gradient3d(*args, dobs.astype(np.float32), misfit_only=True)
    b = O.gradient3d(*args, dobs.astype(np.float64), misfit_only=True)
    assert a[0] == b[0] and a[0] > 0


def test_oracle_linear_in_wavelet_and_zero_source():
    s = S.small3d(nx=24, ny=24, nz=20, nt=70, npad=4, rec_step=4)
    g = s.geom()
    n = s.nxyz
    c = _split(s.cij(), n)
    d1 = O.model_data3d(g, *c, s.wavelet, s.souloc, [0], s.recloc)
    d2 = O.model_data3d(g, *c, 3.0 * s.wavelet, s.souloc, [0], s.recloc)
    # source amplitudes are float products dt2*w (as in the reference)
    assert rel_l2(d2, 3.0 * d1) < 1e-6
    d0 = O.model_data3d(g, *c, 0.0 * s.wavelet, s.souloc, [0], s.recloc)
    assert not d0.any()


def test_oracle_zero_residual_gives_zero_gradient():
    c = K.case3d("g3_a")
    s = c["s"]
    g = s.geom()
    n = s.nxyz
    # observed data from the same model (the sponge pass models with the pad
    # boundary swapped in) and the same code: the residual is exactly 0
    import vtib200 as V
    cp = np.concatenate([V.put_boundary(c["padb"][k * s.nb:(k + 1) * s.nb],
                                        c["cij"][k * n:(k + 1) * n], s.nx, s.ny, s.nz, s.npad)
                         for k in range(3)])
    dobs = O.model_data3d(g, *_split(cp, n), s.wavelet, s.souloc, c["shotid"], s.recloc,
                          dtype=np.float32)
    fg = O.gradient3d(g, c["cij"], c["padb"], c["randb"], s.wavelet, s.souloc, c["shotid"],
                      s.recloc, dobs, dtype=np.float32)
    assert fg[0] == 0.0 and not fg[1:].any()


def test_reference_truncates_levels():
    g = S.small3d(nt=100).geom()
    assert O.last_level(g) == 1 + 64 * ((100 - 2) // 64) == 65
    assert O.last_level(g, full_steps=True) == 99


@pytest.mark.parametrize("name", K.RTM_CASES3D)
def test_oracle_rtm3d_matches_reference(name):
    """rtmCij3d_f restated (FP64) against the reference's own image."""
    c = K.case3d(name)
    s = c["s"]
    g = s.geom()
    n = s.nxyz
    model = K.rtm_model3d(c)
    dobs = load_golden(name)["dobs"]
    gold = load_golden(f"{name}_rtm")
    assert gold["inputs"] == K.digest(s.souloc, s.recloc, s.wavelet, model, dobs)
    o = O.rtm3d(g, *_split(model, n), s.wavelet, s.souloc, c["shotid"], s.recloc, dobs)
    assert np.abs(o).max() > 0
    assert rel_l2(o, gold["image"]) < 1e-4


def test_oracle_odcig3d_zero_lag_is_the_pinned_rtm_image():
    """3D offset gathers (the reference's odcig3d_f target does not link, so
    the gathers are pinned through the RTM image the reference does produce):
    the zero-lag gather of the FP64 restatement is its RTM image bit for bit
    on the imaged x range and zero elsewhere, that image matches the
    reference's, and a trace-free shot gives empty gathers."""
    name = K.RTM_CASES3D[0]
    c = K.case3d(name)
    s = c["s"]
    g = s.geom()
    n = s.nxyz
    model = K.rtm_model3d(c)
    dobs = load_golden(name)["dobs"]
    img = O.rtm3d(g, *_split(model, n), s.wavelet, s.souloc, c["shotid"], s.recloc, dobs)
    assert rel_l2(img, load_golden(f"{name}_rtm")["image"]) < 1e-4
    nlag = 5
    gat = O.odcig3d(g, *_split(model, n), s.wavelet, s.souloc, c["shotid"], s.recloc, dobs, nlag)
    mask = np.zeros((s.nz, s.ny, s.nx), dtype=bool)
    mask[:, :, nlag:s.nx - nlag] = True
    mask = mask.reshape(-1)
    np.testing.assert_array_equal(gat[nlag][mask], img[mask])
    assert not gat[:, ~mask].any()
    assert all(np.abs(gat[k]).max() > 0 for k in range(2 * nlag + 1))
    empty = O.odcig3d(g, *_split(model, n), s.wavelet, s.souloc, c["shotid"], s.recloc,
                      np.zeros_like(dobs), nlag)
    assert not empty.any()


@pytest.mark.parametrize("name", K.RTM_CASES2D)
def test_oracle_rtm2d_matches_reference(name):
    """rtm_f restated (FP64) against the reference's own image."""
    s = K.case2d(name)["s"]
    g = s.geom()
    dobs = load_golden(name)["dobs"]
    gold = load_golden(f"{name}_rtm")
    assert gold["inputs"] == K.digest(s.c11, s.c13, s.c33, s.taper, s.wavelet, s.sloc, s.rloc,
                                      dobs)
    o = O.rtm2d(g, s.c11, s.c13, s.c33, s.wavelet, s.sloc, s.rloc, s.taper, dobs)
    assert np.abs(o).max() > 0
    assert rel_l2(o, gold["image"]) < 1e-4


@pytest.mark.parametrize("name", K.WGRAD_CASES3D)
def test_oracle_wavelet_gradient3d_matches_reference(name):
    """waveletGradientCij3d_f restated (FP64) against the reference's output."""
    c = K.case3d(name)
    s = c["s"]
    g = s.geom()
    n = s.nxyz
    model = K.pad_model3d(c)
    dobs = load_golden(name)["dobs"]
    gold = load_golden(f"{name}_wgrad")
    assert gold["inputs"] == K.digest(s.souloc, s.recloc, model, dobs)
    o = O.wavelet_gradient3d(g, *_split(model, n), s.souloc, c["shotid"], s.recloc, dobs)
    assert np.abs(o).max() > 0
    assert rel_l2(o, gold["gwavelet"]) < 1e-4


@pytest.mark.parametrize("name", K.WGRAD_CASES2D)
def test_oracle_wavelet_gradient2d_matches_reference(name):
    """waveletGradient_f restated (FP64) against the reference's output."""
    s = K.case2d(name)["s"]
    g = s.geom()
    dobs = load_golden(name)["dobs"]
    gold = load_golden(f"{name}_wgrad")
    assert gold["inputs"] == K.digest(s.c11, s.c13, s.c33, s.taper, s.sloc, s.rloc, dobs)
    o = O.wavelet_gradient2d(g, s.c11, s.c13, s.c33, s.sloc, s.rloc, s.taper, dobs)
    assert np.abs(o).max() > 0
    assert rel_l2(o, gold["gwavelet"]) < 1e-4


@pytest.mark.parametrize("name", K.MISFIT_CASES3D)
@pytest.mark.parametrize("key", sorted(K.MISFIT_OPTIONS))
def test_oracle_gradient_misfit_options_match_reference(name, key):
    """tpow gain / AGC misfit of objFuncGradientCij3d_f restated (FP64)."""
    c = K.case3d(name)
    s = c["s"]
    g = s.geom()
    dobs = load_golden(name)["dobs"]
    gold = load_golden(f"{name}_misfit")
    assert gold["inputs"] == K.digest(s.souloc, s.recloc, s.wavelet, c["cij"], c["padb"],
                                      c["randb"], dobs)
    fg = O.gradient3d(g, c["cij"], c["padb"], c["randb"], s.wavelet, s.souloc, c["shotid"],
                      s.recloc, dobs, **K.MISFIT_OPTIONS[key])
    ref = gold[f"fgcij_{key}"].astype(np.float64)
    assert abs(fg[0] - ref[0]) / abs(ref[0]) < 1e-5
    n = s.nxyz
    for k in range(3):
        assert rel_l2(fg[1 + k * n:1 + (k + 1) * n], ref[1 + k * n:1 + (k + 1) * n]) < 1e-4, k


@pytest.mark.parametrize("name", sorted(K.ODCIG_CASES2D))
def test_oracle_odcig2d_matches_reference(name):
    """odcig_f restated (FP64) against the reference's own gathers."""
    s = K.case2d(name)["s"]
    g = s.geom()
    nhx = K.ODCIG_CASES2D[name]
    dobs = load_golden(name)["dobs"]
    gold = load_golden(f"{name}_odcig")
    assert int(gold["nhx"]) == nhx
    assert gold["inputs"] == K.digest(s.c11, s.c13, s.c33, s.taper, s.wavelet, s.sloc, s.rloc,
                                      dobs)
    o = O.odcig2d(g, nhx, s.c11, s.c13, s.c33, s.wavelet, s.sloc, s.rloc, s.taper, dobs)
    assert rel_l2(o.reshape(-1), gold["image"]) < 1e-4
