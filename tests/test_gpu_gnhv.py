"""GPU tests of the exact-mode 3D Gauss-Newton product and gradient
(vti3d_gnhv_exact) against the FP64 oracle's EXACT mode (the operators whose
dot-product and finite-difference tests are in tests/test_exact_adjoint.py).

Tolerances (relative L2): traces 1e-5 (FP32 stencil vs FP64); Born traces,
gradient and H dc 1e-4 (the Born field is driven by products dC L a of an
FP32 wavefield, the images are sums of such products over every level;
measured 2.9e-5 for the Born traces); H dc with the background stored as
BF16 for the imaging: 3e-3 (measured 1.7e-3, 7.6e-4, 9.9e-4 for c11, c13, c33).
"""
import numpy as np
import pytest

import oracle as O
from conftest import rel_l2

import vtib200 as V
import vtib200.synth as S

pytestmark = pytest.mark.gpu

TRACE_TOL = 1e-5
IMG_TOL = 1e-4
# BF16 background (8-bit mantissa, 2^-9 relative rounding per stored value)
BF16_TOL = 3e-3


def _split(a, n):
    return [a[k * n:(k + 1) * n] for k in range(3)]


@pytest.fixture(scope="module")
def case():
    s = S.small3d(nx=52, ny=44, nz=36, nt=150, npad=8, rec_step=3, rate=2.1e-3)
    true = S.small3d(nx=52, ny=44, nz=36, nt=150, npad=8, seed=11)
    n = s.nxyz
    c = s.cij()
    rng = np.random.default_rng(7)
    dc = (rng.standard_normal(3 * n) * c * 1e-2).astype(np.float32)
    dobs = O.exact_forward3d(s.geom(), *_split(true.cij(), n), s.wavelet, s.souloc, [0],
                             s.recloc).astype(np.float32)
    return dict(s=s, g=s.geom(), n=n, c=c, dc=dc, dobs=dobs)


def test_gnhv_matches_exact_oracle(ctx, case):
    s, g, n = case["s"], case["g"], case["n"]
    out = V.gnhv_exact(ctx, g, *_split(case["c"], n), s.wavelet, s.souloc, s.recloc,
                       dc=case["dc"], dobs=case["dobs"], checkpoint_every=16)
    c64 = [a.astype(np.float64) for a in _split(case["c"], n)]
    tr = O.exact_forward3d(g, *c64, s.wavelet, s.souloc, [0], s.recloc)
    bo = O.exact_born3d(g, *c64, s.wavelet, s.souloc, [0], s.recloc, case["dc"])
    assert np.abs(tr).max() > 0 and np.abs(bo).max() > 0
    assert rel_l2(out["traces"], tr) < TRACE_TOL
    assert rel_l2(out["born"], bo) < IMG_TOL
    r = tr - case["dobs"]
    assert abs(out["misfit"] - 0.5 * r @ r) / (0.5 * r @ r) < 1e-4
    gr = O.exact_adjoint3d(g, *c64, s.wavelet, s.souloc, [0], s.recloc, r)
    hv = O.exact_adjoint3d(g, *c64, s.wavelet, s.souloc, [0], s.recloc, bo)
    for k, (a, b) in enumerate(zip(_split(out["grad"], n), _split(gr, n))):
        assert np.abs(b).max() > 0
        assert rel_l2(a, b) < IMG_TOL, ("grad", k)
    for k, (a, b) in enumerate(zip(_split(out["hv"], n), _split(hv, n))):
        assert np.abs(b).max() > 0
        assert rel_l2(a, b) < IMG_TOL, ("hv", k)


def test_gnhv_checkpoint_interval_and_symmetry(ctx, case):
    """The recomputation reproduces the forward levels: any checkpoint
    interval gives the same product; H is symmetric (<u, H v> = <v, H u>)."""
    s, g, n = case["s"], case["g"], case["n"]
    cs = _split(case["c"], n)
    h1 = V.gnhv_exact(ctx, g, *cs, s.wavelet, s.souloc, s.recloc, dc=case["dc"],
                      checkpoint_every=5, want=("hv",))["hv"]
    h2 = V.gnhv_exact(ctx, g, *cs, s.wavelet, s.souloc, s.recloc, dc=case["dc"],
                      checkpoint_every=1000, want=("hv",))["hv"]
    assert rel_l2(h1, h2) < 1e-6
    rng = np.random.default_rng(9)
    u = (rng.standard_normal(3 * n) * case["c"] * 1e-2).astype(np.float32)
    hu = V.gnhv_exact(ctx, g, *cs, s.wavelet, s.souloc, s.recloc, dc=u, want=("hv",))["hv"]
    a = float(np.dot(case["dc"].astype(np.float64), hu))
    b = float(np.dot(u.astype(np.float64), h1))
    assert abs(a - b) / abs(a) < 1e-4
    # Gauss-Newton Hessian is positive semi-definite
    assert float(np.dot(case["dc"].astype(np.float64), h1)) > 0


def test_gnhv_bf16_background(ctx, case):
    """BF16 storage (per-plane scales) of the background levels the imaging
    reads: the images stay within the stated error of the FP64 oracle; the
    traces are unchanged (the forward pass and checkpoints stay FP32)."""
    s, g, n = case["s"], case["g"], case["n"]
    cs = _split(case["c"], n)
    f32 = V.gnhv_exact(ctx, g, *cs, s.wavelet, s.souloc, s.recloc, dc=case["dc"],
                       dobs=case["dobs"], checkpoint_every=16)
    b16 = V.gnhv_exact(ctx, g, *cs, s.wavelet, s.souloc, s.recloc, dc=case["dc"],
                       dobs=case["dobs"], checkpoint_every=16, flags=V.GNHV_BF16)
    np.testing.assert_array_equal(b16["traces"], f32["traces"])
    np.testing.assert_array_equal(b16["born"], f32["born"])
    assert b16["misfit"] == f32["misfit"]
    c64 = [a.astype(np.float64) for a in cs]
    bo = O.exact_born3d(g, *c64, s.wavelet, s.souloc, [0], s.recloc, case["dc"])
    hv = O.exact_adjoint3d(g, *c64, s.wavelet, s.souloc, [0], s.recloc, bo)
    errs = [rel_l2(a, b) for a, b in zip(_split(b16["hv"], n), _split(hv, n))]
    print("BF16 background (round to nearest): H dc rel-L2 vs FP64", errs)
    assert max(errs) < BF16_TOL
    # stochastic rounding: unbiased values, but twice the per-value variance;
    # here the round-to-nearest errors do not add coherently, so it is about
    # twice as far from FP64 (measured 3.1e-3, 1.7e-3, 1.6e-3)
    sr = V.gnhv_exact(ctx, g, *cs, s.wavelet, s.souloc, s.recloc, dc=case["dc"],
                      dobs=case["dobs"], checkpoint_every=16, flags=V.GNHV_BF16 | V.GNHV_BF16_SR)
    errs_sr = [rel_l2(a, b) for a, b in zip(_split(sr["hv"], n), _split(hv, n))]
    print("BF16 background (stochastic rounding): H dc rel-L2 vs FP64", errs_sr)
    assert max(errs_sr) < 2 * BF16_TOL
    np.testing.assert_array_equal(sr["traces"], f32["traces"])
