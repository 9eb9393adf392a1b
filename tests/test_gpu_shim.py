"""Drop-in test: the harness that drives the reference's own entry points
(oracle/ref_driver{3d,2d}.cpp: modelDataCij3d_f, objFuncGradientCij3d_f with
the data= side channel, synthetic_f, modeling_f) is compiled against
libvti_wave.so instead of the reference objects, and must reproduce the
reference's golden outputs."""
import subprocess
import tempfile
from pathlib import Path

import numpy as np
import pytest

import cases as K
import make_golden as MG
from conftest import ROOT, load_golden, rel_l2

pytestmark = pytest.mark.gpu

LIBDIR = ROOT / "thesis-source-code_b200" / "vtib200"


@pytest.fixture(scope="module")
def drivers(tmp_path_factory):
    out = tmp_path_factory.mktemp("shim")
    bins = {}
    for dim in ("3d", "2d"):
        exe = out / f"shim{dim}"
        subprocess.run(
            ["g++", "-O2", "-std=c++17", "-DVTI_SHIM",
             str(ROOT / "oracle" / f"ref_driver{dim}.cpp"),
             str(ROOT / "tests" / "shim" / "myio_stub.cpp"), "-I", str(ROOT / "include"),
             f"-L{LIBDIR}", "-lvti_wave", "-lvti_b200", f"-Wl,-rpath,{LIBDIR}", "-o", str(exe)],
            check=True)
        bins[dim] = exe
    return bins


def _run(exe, d, mode, *params):
    r = subprocess.run([str(exe), str(d), mode, *params], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]


@pytest.mark.parametrize("name", K.GRAD_CASES3D)
def test_shim_3d_matches_reference(drivers, name):
    c = K.case3d(name)
    gold = load_golden(name)
    with tempfile.TemporaryDirectory() as td:
        d = Path(td)
        MG.write_inputs3d(c, d)
        np.asarray(c["cij_true"], np.float32).tofile(d / "cij.bin")
        _run(drivers["3d"], d, "model")
        dobs = np.fromfile(d / "ref_ddata.bin", dtype=np.float32)
        assert rel_l2(dobs, gold["dobs"]) < 1e-5
        np.asarray(gold["dobs"], np.float32).tofile(d / "dobs.bin")
        np.asarray(c["cij"], np.float32).tofile(d / "cij.bin")
        _run(drivers["3d"], d, "grad")
        fg = np.fromfile(d / "ref_fgcij.bin", dtype=np.float32)
    ref = gold["fgcij"]
    assert abs(fg[0] - ref[0]) / ref[0] < 1e-5
    n = (ref.size - 1) // 3
    for k in range(3):
        assert rel_l2(fg[1 + k * n:1 + (k + 1) * n], ref[1 + k * n:1 + (k + 1) * n]) < 1e-4


@pytest.mark.parametrize("name", K.CASES2D)
def test_shim_2d_matches_reference(drivers, name):
    s = K.case2d(name)["s"]
    gold = load_golden(name)
    with tempfile.TemporaryDirectory() as td:
        d = Path(td)
        MG.write_inputs2d(s, d)
        _run(drivers["2d"], d, "synthetic")
        data = np.fromfile(d / "ref_data.bin", dtype=np.float32)
        _run(drivers["2d"], d, "modeling")
        w = np.fromfile(d / "ref_wavefield.bin", dtype=np.float32)
        # objFuncGradient_f and GNhessian_f at the starting model
        np.asarray(gold["dobs"], np.float32).tofile(d / "data.bin")
        c = K.case2d(name)
        for k in ("c11", "c13", "c33"):
            c["dc"][k].tofile(d / f"d{k}.bin")
        _run(drivers["2d"], d, "grad")
        grad = np.fromfile(d / "ref_grad.bin", dtype=np.float32)
        _run(drivers["2d"], d, "gnhess")
        gnh = np.fromfile(d / "ref_gnhess.bin", dtype=np.float32)
        # the Gauss-Newton operator classes (HessianOp.h) through the shim
        _run(drivers["2d"], d, "gnhessop")
        op = np.fromfile(d / "ref_gnhessop.bin", dtype=np.float32)
    assert rel_l2(data, gold["data"]) < 1e-5
    nnxz = (s.nx + 2 * s.npad) * (s.nz + 2 * s.npad)
    w = w.reshape(-1, nnxz)
    assert rel_l2(w[gold["snap_rows"]], gold["snaps"]) < 3e-5
    ref = gold["grad"]
    assert abs(grad[3 * nnxz] - ref[3 * nnxz]) / ref[3 * nnxz] < 1e-5
    for k in range(3):
        sl = slice(k * nnxz, (k + 1) * nnxz)
        assert rel_l2(grad[sl], ref[sl]) < 1e-4, k
        assert rel_l2(gnh[sl], gold["gnhess"][sl]) < 1e-4, k
        # GNHessianOpCij: GNhessianCij (scales 1) = GNhessian_f with the pad
        # rows (npad + 0/dz + 1) zeroed; adjoint(add) doubles it
        ref_op = np.array(gold["gnhess"][sl], dtype=np.float32).reshape(-1, s.nx + 2 * s.npad)
        ref_op[:s.npad + 1] = 0
        assert rel_l2(op[sl], ref_op.reshape(-1)) < 1e-4, k
        np.testing.assert_array_equal(op[3 * nnxz + k * nnxz:3 * nnxz + (k + 1) * nnxz],
                                      2 * op[sl])


@pytest.mark.parametrize("name", K.RTM_CASES3D)
def test_shim_rtm3d_matches_reference(drivers, name):
    """rtmCij3d_f through the drop-in library (three floats per receiver, the
    traces read from data=) against the reference's own image."""
    c = K.case3d(name)
    with tempfile.TemporaryDirectory() as td:
        d = Path(td)
        MG.write_inputs3d(c, d)
        K.rtm_model3d(c).astype(np.float32).tofile(d / "cij.bin")
        np.asarray(load_golden(name)["dobs"], np.float32).tofile(d / "dobs.bin")
        _run(drivers["3d"], d, "rtm")
        img = np.fromfile(d / "ref_image.bin", dtype=np.float32)
    assert rel_l2(img, load_golden(f"{name}_rtm")["image"]) < 1e-4


@pytest.mark.parametrize("name", K.RTM_CASES2D)
def test_shim_rtm2d_matches_reference(drivers, name):
    s = K.case2d(name)["s"]
    with tempfile.TemporaryDirectory() as td:
        d = Path(td)
        MG.write_inputs2d(s, d)
        np.asarray(load_golden(name)["dobs"], np.float32).tofile(d / "data.bin")
        _run(drivers["2d"], d, "rtm")
        img = np.fromfile(d / "ref_rtm.bin", dtype=np.float32)
    assert rel_l2(img, load_golden(f"{name}_rtm")["image"]) < 1e-4


@pytest.mark.parametrize("name", K.WGRAD_CASES3D)
def test_shim_wavelet_gradient3d_matches_reference(drivers, name):
    c = K.case3d(name)
    with tempfile.TemporaryDirectory() as td:
        d = Path(td)
        MG.write_inputs3d(c, d)
        K.pad_model3d(c).astype(np.float32).tofile(d / "cij.bin")
        np.asarray(load_golden(name)["dobs"], np.float32).tofile(d / "dobs.bin")
        _run(drivers["3d"], d, "wgrad")
        gw = np.fromfile(d / "ref_wgrad.bin", dtype=np.float32)
    assert rel_l2(gw, load_golden(f"{name}_wgrad")["gwavelet"]) < 1e-4


@pytest.mark.parametrize("name", K.WGRAD_CASES3D)
def test_shim_modeling_operator3d(drivers, name):
    """ModelingOp3d (ModelingOp3d.cu:12-33) from the reference's header layout:
    forward = modelData3d_f of the wavelet (the reference's traces), adjoint =
    waveletGradient3d_f (the reference's wavelet gradient), add accumulates."""
    c = K.case3d(name)
    gold = load_golden(name)
    with tempfile.TemporaryDirectory() as td:
        d = Path(td)
        MG.write_inputs3d(c, d)
        np.asarray(gold["dobs"], np.float32).tofile(d / "dobs.bin")
        np.asarray(c["cij_true"], np.float32).tofile(d / "cij.bin")
        _run(drivers["3d"], d, "model")
        _run(drivers["3d"], d, "modop")
        ddata = np.fromfile(d / "ref_ddata.bin", dtype=np.float32)
        fwd = np.fromfile(d / "ref_modop_fwd.bin", dtype=np.float32)
        fwd_add = np.fromfile(d / "ref_modop_fwd_add.bin", dtype=np.float32)
        K.pad_model3d(c).astype(np.float32).tofile(d / "cij.bin")
        _run(drivers["3d"], d, "modop")
        adj = np.fromfile(d / "ref_modop_adj.bin", dtype=np.float32)
        adj_add = np.fromfile(d / "ref_modop_adj_add.bin", dtype=np.float32)
    np.testing.assert_array_equal(fwd, ddata)
    assert rel_l2(fwd, gold["dobs"]) < 1e-5
    np.testing.assert_array_equal(fwd_add, np.float32(1) + fwd)
    assert adj.size == c["s"].nt
    assert rel_l2(adj, load_golden(f"{name}_wgrad")["gwavelet"]) < 1e-4
    np.testing.assert_array_equal(adj_add, np.float32(1) + adj)


@pytest.mark.parametrize("name", K.WGRAD_CASES2D)
def test_shim_wavelet_gradient2d_matches_reference(drivers, name):
    s = K.case2d(name)["s"]
    with tempfile.TemporaryDirectory() as td:
        d = Path(td)
        MG.write_inputs2d(s, d)
        np.asarray(load_golden(name)["dobs"], np.float32).tofile(d / "data.bin")
        _run(drivers["2d"], d, "wgrad")
        gw = np.fromfile(d / "ref_wgrad.bin", dtype=np.float32)
    assert rel_l2(gw, load_golden(f"{name}_wgrad")["gwavelet"]) < 1e-4


@pytest.mark.parametrize("name", K.MISFIT_CASES3D)
@pytest.mark.parametrize("key", sorted(K.MISFIT_OPTIONS))
def test_shim_gradient_misfit_options_match_reference(drivers, name, key):
    """tpow= / objtype= / halfwidth= read from the caller's argv."""
    c = K.case3d(name)
    opt = K.MISFIT_OPTIONS[key]
    with tempfile.TemporaryDirectory() as td:
        d = Path(td)
        MG.write_inputs3d(c, d)
        np.asarray(load_golden(name)["dobs"], np.float32).tofile(d / "dobs.bin")
        np.asarray(c["cij"], np.float32).tofile(d / "cij.bin")
        _run(drivers["3d"], d, "grad", *[f"{k}={v}" for k, v in opt.items()])
        fg = np.fromfile(d / "ref_fgcij.bin", dtype=np.float32)
    ref = load_golden(f"{name}_misfit")[f"fgcij_{key}"]
    assert abs(fg[0] - ref[0]) / ref[0] < 1e-5
    n = (ref.size - 1) // 3
    for k in range(3):
        assert rel_l2(fg[1 + k * n:1 + (k + 1) * n], ref[1 + k * n:1 + (k + 1) * n]) < 1e-4


@pytest.mark.parametrize("name", sorted(K.ODCIG_CASES2D))
def test_shim_odcig2d_matches_reference(drivers, name):
    s = K.case2d(name)["s"]
    with tempfile.TemporaryDirectory() as td:
        d = Path(td)
        MG.write_inputs2d(s, d)
        np.asarray(load_golden(name)["dobs"], np.float32).tofile(d / "data.bin")
        _run(drivers["2d"], d, "odcig", str(K.ODCIG_CASES2D[name]))
        img = np.fromfile(d / "ref_odcig.bin", dtype=np.float32)
    assert rel_l2(img, load_golden(f"{name}_odcig")["image"]) < 1e-4


def test_shim_odcig3d_matches_the_plan(drivers, ctx):
    """odcig3d_f through the drop-in (the reference's own target does not
    link): v, eps, del derived from c_ij by the harness, 32 lags, equal to
    the plan's gathers of the same model within the image tolerance (the
    v/eps/del round trip moves c_ij by a few ulps)."""
    import vtib200 as V
    import vtib200.synth as S
    s = S.small3d(nx=80, ny=28, nz=24, nt=110, npad=6, rec_step=3, rate=2.1e-3)
    true = S.small3d(nx=80, ny=28, nz=24, nt=110, npad=6, seed=11)
    g = s.geom()
    n = s.nxyz
    padb, randb = S.boundaries3d(s)
    tc = true.cij()
    dobs = V.modelDataCij3d_f(ctx, g, s.souloc, [0], s.recloc, s.wavelet, tc[:n], tc[n:2 * n],
                              tc[2 * n:])
    model = s.cij()
    with tempfile.TemporaryDirectory() as td:
        d = Path(td)
        MG.write_inputs3d({"s": s, "padb": padb, "randb": randb}, d)
        np.asarray(model, np.float32).tofile(d / "cij.bin")
        np.asarray(dobs, np.float32).tofile(d / "dobs.bin")
        _run(drivers["3d"], d, "odcig")
        shim = np.fromfile(d / "ref_odcig.bin", dtype=np.float32).reshape(65, n)
    p = V.Plan3d(ctx, g)
    try:
        p.set_model(model[:n], model[n:2 * n], model[2 * n:])
        p.set_wavelet(s.wavelet)
        p.set_receivers(s.recloc)
        gat = p.odcig(s.souloc, [0], dobs, 32)
    finally:
        p.close()
    assert np.abs(gat[32]).max() > 0
    assert rel_l2(shim.reshape(-1), gat.reshape(-1)) < 1e-4
