"""GPU parity tests of the 3D path, called through the C ABI.

Tolerances (relative L2): FP32 traces 1e-5 against the FP64 oracle and the
reference's own outputs; gradients 1e-4 against the FP64 oracle.
"""
import numpy as np
import pytest

import cases as K
import oracle as O
from conftest import load_golden, rel_l2

import vtib200 as V
import vtib200.synth as S

pytestmark = pytest.mark.gpu

TRACE_TOL = 1e-5
GRAD_TOL = 1e-4


def _split(cij, n):
    return cij[:n], cij[n:2 * n], cij[2 * n:]


def _parts(fg, n):
    return [fg[1 + k * n:1 + (k + 1) * n] for k in range(3)]


@pytest.mark.parametrize("name", K.CASES3D)
def test_model_data_matches_oracle_and_reference(ctx, name):
    c = K.case3d(name)
    s = c["s"]
    g = s.geom()
    n = s.nxyz
    d = V.modelDataCij3d_f(ctx, g, s.souloc, c["shotid"], s.recloc, s.wavelet,
                           *_split(c["cij_true"], n))
    o = O.model_data3d(g, *_split(c["cij_true"], n), s.wavelet, s.souloc, c["shotid"], s.recloc)
    assert np.abs(o).max() > 0
    assert rel_l2(d, o) < TRACE_TOL
    gold = load_golden(name)
    assert np.abs(gold["dobs"]).max() > 0
    assert rel_l2(d, gold["dobs"]) < TRACE_TOL
    # the same samples are recorded (and left at zero) as by the reference
    assert np.array_equal(d != 0, gold["dobs"] != 0)


@pytest.mark.parametrize("name", K.GRAD_CASES3D)
def test_gradient_matches_oracle_and_reference(ctx, name):
    c = K.case3d(name)
    s = c["s"]
    g = s.geom()
    n = s.nxyz
    gold = load_golden(name)
    dobs = gold["dobs"]
    fg, mis = V.objFuncGradientCij3d_f(ctx, g, s.souloc, c["shotid"], s.recloc, s.wavelet,
                                       c["cij"], c["padb"], c["randb"], dobs)
    o = O.gradient3d(g, c["cij"], c["padb"], c["randb"], s.wavelet, s.souloc, c["shotid"],
                     s.recloc, dobs)
    assert abs(mis - o[0]) / o[0] < TRACE_TOL
    assert abs(fg[0] - o[0]) / o[0] < TRACE_TOL
    ref = gold["fgcij"]
    assert abs(fg[0] - ref[0]) / ref[0] < TRACE_TOL
    for k, (a, b, r) in enumerate(zip(_parts(fg, n), _parts(o, n), _parts(ref, n))):
        assert np.abs(b).max() > 0 and np.abs(r).max() > 0
        assert rel_l2(a, b) < GRAD_TOL, k
        assert rel_l2(a, r) < GRAD_TOL, k


def test_odd_grid_matches_oracle(ctx):
    """Odd nx and ny: the last tile column and row are partly outside the
    update region, and x = nx-5 is updated while its neighbour nx-4 is not."""
    s = S.small3d(nx=45, ny=39, nz=30, nt=110, npad=6, rec_step=3, rate=2.1e-3)
    true = S.small3d(nx=45, ny=39, nz=30, nt=110, npad=6, seed=11)
    g = s.geom()
    n = s.nxyz
    shot = [0]
    padb, randb = S.boundaries3d(s)
    dobs = V.modelDataCij3d_f(ctx, g, s.souloc, shot, s.recloc, s.wavelet, *_split(true.cij(), n))
    od = O.model_data3d(g, *_split(true.cij(), n), s.wavelet, s.souloc, shot, s.recloc)
    assert np.abs(od).max() > 0
    assert rel_l2(dobs, od) < TRACE_TOL
    fg, mis = V.objFuncGradientCij3d_f(ctx, g, s.souloc, shot, s.recloc, s.wavelet, s.cij(), padb,
                                       randb, od)
    o, mod = O.gradient3d(g, s.cij(), padb, randb, s.wavelet, s.souloc, shot, s.recloc, od,
                          want_modeled=True)
    # the misfit of a small residual r carries the trace error magnified:
    # |dJ|/J <= 2 * TRACE_TOL * |d| / |r| to first order (|r|/|d| is ~6 % here)
    mis_tol = 2 * TRACE_TOL * np.linalg.norm(od) / np.linalg.norm(mod - od)
    assert abs(mis - o[0]) / o[0] < mis_tol
    for k, (a, b) in enumerate(zip(_parts(fg, n), _parts(o, n))):
        assert np.abs(b).max() > 0
        assert rel_l2(a, b) < GRAD_TOL, k


def test_full_steps_option(ctx):
    c = K.case3d("g3_b")
    s = c["s"]
    g = s.geom()
    n = s.nxyz
    d = V.modelDataCij3d_f(ctx, g, s.souloc, c["shotid"], s.recloc, s.wavelet,
                           *_split(c["cij"], n), flags=V.OPT_FULL_STEPS)
    o = O.model_data3d(g, *_split(c["cij"], n), s.wavelet, s.souloc, c["shotid"], s.recloc,
                       full_steps=True)
    assert rel_l2(d, o) < TRACE_TOL
    # the reference truncation leaves the late samples at zero
    nnt = O.nnt3d(g)
    tr = O.model_data3d(g, *_split(c["cij"], n), s.wavelet, s.souloc, c["shotid"], s.recloc)
    assert not tr.reshape(-1, nnt)[:, O.last_level(g) // 2 + 1:].any()
    assert np.abs(o.reshape(-1, nnt)[:, -5:]).max() > 0


def test_plan_reuse_is_deterministic_and_objfunc_agrees(ctx):
    c = K.case3d("g3_a")
    s = c["s"]
    g = s.geom()
    n = s.nxyz
    gold = load_golden("g3_a")
    p = V.Plan3d(ctx, g)
    try:
        p.set_model(*_split(c["cij"], n), padb=c["padb"], randb=c["randb"])
        p.set_wavelet(s.wavelet)
        p.set_receivers(s.recloc)
        fg1, m1 = p.gradient(s.souloc, c["shotid"], gold["dobs"])
        fg2, m2 = p.gradient(s.souloc, c["shotid"], gold["dobs"])
        np.testing.assert_array_equal(fg1, fg2)
        assert m1 == m2
        m3 = p.objfunc(s.souloc, c["shotid"], gold["dobs"])
        assert m3 == m1
    finally:
        p.close()


def test_one_call_forms_keep_no_state_between_calls(ctx):
    """The context keeps the plan of the one-call forms while the geometry and
    flags repeat (gradient with a random boundary, modeling without one,
    another model): every output equals that of calls with their own plan."""
    c = K.case3d("g3_a")
    s = c["s"]
    g = s.geom()
    n = s.nxyz
    dobs = load_golden("g3_a")["dobs"]

    def run():
        fa, ma = V.objFuncGradientCij3d_f(ctx, g, s.souloc, c["shotid"], s.recloc, s.wavelet,
                                          c["cij"], c["padb"], c["randb"], dobs)
        d = V.modelDataCij3d_f(ctx, g, s.souloc, c["shotid"], s.recloc, s.wavelet,
                               *_split(c["cij_true"], n))
        fb, mb = V.objFuncGradientCij3d_f(ctx, g, s.souloc, c["shotid"], s.recloc, s.wavelet,
                                          c["cij_true"], c["padb"], c["randb"], dobs)
        return fa, ma, d, fb, mb

    kept = run()
    again = run()
    ctx.set_plan_cache(False)
    try:
        fresh = run()
    finally:
        ctx.set_plan_cache(True)
    assert np.abs(kept[2]).max() > 0 and kept[1] > 0 and kept[4] != kept[1]
    for a, b, r in zip(kept, again, fresh):
        np.testing.assert_array_equal(a, r)
        np.testing.assert_array_equal(b, r)


def test_one_call_plan_follows_the_geometry(ctx):
    """A one-call form with another geometry (or flags) replaces the kept
    plan; going back to the first geometry gives its results again."""
    def case(nt):
        s = S.small3d(nx=40, ny=36, nz=28, nt=nt, npad=6, rec_step=3, rate=2.1e-3)
        true = S.small3d(nx=40, ny=36, nz=28, nt=nt, npad=6, seed=11)
        return s, true

    def run(s, true, flags):
        n = s.nxyz
        g = s.geom()
        padb, randb = S.boundaries3d(s)
        d = V.modelDataCij3d_f(ctx, g, s.souloc, [0], s.recloc, s.wavelet,
                               *_split(true.cij(), n), flags=flags)
        fg, mis = V.objFuncGradientCij3d_f(ctx, g, s.souloc, [0], s.recloc, s.wavelet, s.cij(),
                                           padb, randb, d, flags=flags)
        return d, fg, mis

    a, b = case(110), case(90)
    seq = [(a, 0), (b, 0), (a, V.OPT_FULL_STEPS), (a, 0)]
    kept = [run(*c, f) for c, f in seq]
    ctx.set_plan_cache(False)
    try:
        fresh = [run(*c, f) for c, f in seq]
    finally:
        ctx.set_plan_cache(True)
    for k, r in zip(kept, fresh):
        assert np.abs(r[0]).max() > 0 and r[2] > 0
        for u, v in zip(k, r):
            np.testing.assert_array_equal(u, v)
    np.testing.assert_array_equal(kept[0][1], kept[3][1])


def test_zero_residual_gives_zero_gradient(ctx):
    """Observed data modeled by the library itself: residual and gradient are 0."""
    s = S.small3d(nx=72, ny=64, nz=48, nt=130, npad=8, rec_step=2)
    g = s.geom()
    n = s.nxyz
    padb, randb = S.boundaries3d(s)
    cp = np.concatenate([V.put_boundary(padb[k * s.nb:(k + 1) * s.nb], s.cij()[k * n:(k + 1) * n],
                                        s.nx, s.ny, s.nz, s.npad) for k in range(3)])
    dobs = V.modelDataCij3d_f(ctx, g, s.souloc, [0], s.recloc, s.wavelet, *_split(cp, n))
    assert np.abs(dobs).max() > 0
    fg, mis = V.objFuncGradientCij3d_f(ctx, g, s.souloc, [0], s.recloc, s.wavelet, s.cij(), padb,
                                       randb, dobs)
    assert mis == 0.0 and fg[0] == 0.0 and not fg[1:].any()


def test_linearity_in_wavelet_large(ctx):
    """Size-independent property at a larger grid: traces scale with the source."""
    s = S.small3d(nx=160, ny=144, nz=96, nt=194, npad=16, rec_step=4, d=12.5, dt=8e-4,
                  rate=1.6e-3)
    g = s.geom()
    c = _split(s.cij(), s.nxyz)
    d1 = V.modelDataCij3d_f(ctx, g, s.souloc, [0], s.recloc, s.wavelet, *c)
    d2 = V.modelDataCij3d_f(ctx, g, s.souloc, [0], s.recloc, -2.0 * s.wavelet, *c)
    assert np.abs(d1).max() > 0
    assert rel_l2(d2, -2.0 * d1) < 1e-6


def test_source_outside_update_region_is_rejected(ctx):
    s = S.small3d(nx=24, ny=24, nz=20, nt=70, npad=4, rec_step=4)
    g = s.geom()
    so = s.souloc.copy()
    so[0] = s.o + 1.25 * s.d  # ix = 1 lies in the never-updated 4-cell frame
    with pytest.raises(V.VtiError) as e:
        V.modelDataCij3d_f(ctx, g, so, [0], s.recloc, s.wavelet, *_split(s.cij(), s.nxyz))
    assert e.value.status == V.VTI_ERR_ARG
    bad = V.geom3d(8, 8, 8, 10, 2, 10.0, 10.0, 10.0, 1e-3, 2e-3)
    with pytest.raises(V.VtiError):
        V.Plan3d(ctx, bad)


@pytest.mark.parametrize("name", K.MISFIT_CASES3D)
@pytest.mark.parametrize("key", sorted(K.MISFIT_OPTIONS))
def test_gradient_misfit_options_match_oracle_and_reference(ctx, name, key):
    """tpow gain and AGC misfit of the gradient (objFuncGradient3d_f.cu:743-773)."""
    c = K.case3d(name)
    s = c["s"]
    g = s.geom()
    n = s.nxyz
    opt = K.MISFIT_OPTIONS[key]
    dobs = load_golden(name)["dobs"]
    p = V.Plan3d(ctx, g)
    try:
        p.set_model(*_split(c["cij"], n), padb=c["padb"], randb=c["randb"])
        p.set_wavelet(s.wavelet)
        p.set_receivers(s.recloc)
        p.set_misfit(**opt)
        fg, mis = p.gradient(s.souloc, c["shotid"], dobs)
        # the misfit-only entry stays plain L2, like objFuncCij3d_f
        plain = p.objfunc(s.souloc, c["shotid"], dobs)
    finally:
        p.close()
    o = O.gradient3d(g, c["cij"], c["padb"], c["randb"], s.wavelet, s.souloc, c["shotid"],
                     s.recloc, dobs, **opt)
    ref = load_golden(f"{name}_misfit")[f"fgcij_{key}"]
    assert abs(mis - o[0]) / o[0] < TRACE_TOL
    assert abs(fg[0] - ref[0]) / ref[0] < TRACE_TOL
    for k, (a, b, r) in enumerate(zip(_parts(fg, n), _parts(o, n), _parts(ref, n))):
        assert np.abs(b).max() > 0
        assert rel_l2(a, b) < GRAD_TOL, k
        assert rel_l2(a, r) < GRAD_TOL, k
    l2 = O.gradient3d(g, c["cij"], c["padb"], c["randb"], s.wavelet, s.souloc, c["shotid"],
                      s.recloc, dobs, misfit_only=True)
    assert abs(plain - l2[0]) / l2[0] < TRACE_TOL


def test_f16_traces_in_flight(ctx):
    """Observed traces passed as a VTI_TRACES_F16 block (FP16 values, one FP32
    scale per time sample): the plan expands each shot's traces on the device
    to exactly the FP32 traces the block stands for, from host or device
    memory, so the gradient is bitwise that of those traces and within the
    FP32 bar of the FP64 oracle run on them. Against the gradient of the
    original FP32 traces it moves by the quantisation of the data relative to
    the residual (the gradient is linear in the residual): here the residual
    is 13 % of the data and the move is 1e-3."""
    import torch
    c = K.case3d("g3_a")
    s = c["s"]
    g = s.geom()
    n = s.nxyz
    gold = load_golden("g3_a")
    nnt = O.nnt3d(g)
    nr = s.recloc.size // 4
    dobs = np.asarray(gold["dobs"], dtype=np.float32)
    block = V.pack_traces_f16(dobs, nnt)
    assert block.nbytes < 0.51 * dobs.nbytes + 4 * nnt
    dq = V.unpack_traces_f16(block, nr, nnt)
    assert 0 < rel_l2(dq, dobs) < 1e-3
    p = V.Plan3d(ctx, g)
    try:
        p.set_model(*_split(c["cij"], n), padb=c["padb"], randb=c["randb"])
        p.set_wavelet(s.wavelet)
        p.set_receivers(s.recloc)
        fq, mq = p.gradient(s.souloc, c["shotid"], dq)
        iq = p.rtm(s.souloc, c["shotid"], dq)
        p.set_trace_format(V.TRACES_F16)
        fh, mh = p.gradient(s.souloc, c["shotid"], block)
        ih = p.rtm(s.souloc, c["shotid"], block)
        bd = torch.from_numpy(block).cuda()
        fd, md = p.gradient(s.souloc, c["shotid"], bd.data_ptr(), V.MEM_DEVICE)
        torch.cuda.synchronize()
        with pytest.raises(V.VtiError):
            p.set_trace_format(5)
    finally:
        p.close()
    np.testing.assert_array_equal(fh, fq)
    np.testing.assert_array_equal(fd, fq)
    np.testing.assert_array_equal(ih, iq)
    assert mh == mq and md == mq
    oq = O.gradient3d(g, c["cij"], c["padb"], c["randb"], s.wavelet, s.souloc, c["shotid"],
                      s.recloc, dq)
    for a, b in zip(_parts(fh, n), _parts(oq, n)):
        assert np.abs(b).max() > 0
        assert rel_l2(a, b) < GRAD_TOL
    o = O.gradient3d(g, c["cij"], c["padb"], c["randb"], s.wavelet, s.souloc, c["shotid"],
                     s.recloc, dobs)
    mod = O.model_data3d(g, *_split(c["cij"], n), s.wavelet, s.souloc, c["shotid"], s.recloc)
    bound = np.linalg.norm(dq - dobs) / np.linalg.norm(mod - dobs)
    for a, b in zip(_parts(fh, n), _parts(o, n)):
        assert rel_l2(a, b) < 1.5 * bound + GRAD_TOL
