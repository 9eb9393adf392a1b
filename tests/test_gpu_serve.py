"""GPU tests of the serving loop (vtib200.serve): mixed 2D/3D modeling and
gradient requests with continuous batching of the 3D ones, and an FWI driver
whose gradients come from the engine, checked against the plain per-shot
form (vti3d_plan_gradient, objFuncGradient3d_f.cu:361)."""
import numpy as np
import pytest

import vtib200 as V
import vtib200.serve as SV
import vtib200.synth as S

pytestmark = pytest.mark.gpu


def test_mixed_requests_all_served():
    reqs = SV.make_requests(8, rate=200.0, seed=3, size3d=((40, 40, 32), (72, 64, 48)),
                            size2d=((40, 60), (64, 100)), nt=(150, 260), freq=(20.0, 30.0))
    srv = SV.Server(max_bytes=4 << 30, chunk=8)
    try:
        stats = srv.run(reqs, t_limit=600.0)
    finally:
        srv.close()
    assert stats["done"] == len(reqs)
    assert 0 < stats["p50_s"] <= stats["p99_s"]
    for r in reqs:
        assert r.t_done >= r.arrival
        if r.dim == 3:
            out = r.result[0]
            assert np.isfinite(out).all() and np.abs(out).max() > 0


def _fwi_case():
    s = S.small3d(nx=84, ny=76, nz=36, nt=140, npad=8, rate=2.1e-3)
    true = S.small3d(nx=84, ny=76, nz=36, nt=140, npad=8, seed=11)
    g = s.geom()
    n = s.nxyz
    wins = [(0, 0, 56, 52), (28, 24, 56, 52)]
    souloc, recloc = S.batch_survey3d(s, wins, rec_step=3)
    shots = []
    ctx = V.Context(0)
    try:
        for k, (x0, y0, wx, wy) in enumerate(wins):
            so = souloc[5 * k:5 * k + 5].copy()
            nr, first = int(so[3]), int(so[4])
            rec = recloc[4 * first:4 * (first + nr)].copy()
            so[4] = 0
            sub = V.geom3d(wx, wy, g.nz, g.nt, g.npad, g.dx, g.dy, g.dz, g.dt, g.sampling_rate,
                           ox=g.ox + x0 * g.dx, oy=g.oy + y0 * g.dy, oz=g.oz)
            p = V.Plan3d(ctx, sub, V.OPT_FULL_STEPS)
            try:
                ct = true.cij().reshape(3, g.nz, g.ny, g.nx)[:, :, y0:y0 + wy, x0:x0 + wx]
                p.set_model(*[c.reshape(-1) for c in ct])
                p.set_wavelet(s.wavelet)
                p.set_receivers(rec)
                dobs = p.model_data(so, [0])
            finally:
                p.close()
            shots.append((so, rec, dobs, (x0, y0, wx, wy)))
    finally:
        ctx.close()
    c0 = s.cij()
    return g, c0, s.wavelet, shots, float(np.abs(c0).max() * 2e-3)


def test_fwi_in_the_server_matches_the_plain_form():
    """L-BFGS iterations whose gradients come through the engine (beside
    other requests) follow exactly the plain per-shot form's trajectory."""
    g, c0, w, shots, step0 = _fwi_case()
    fwi = SV.FwiDriver(g, c0, w, shots, iterations=2, step0=step0)
    reqs = SV.make_requests(4, rate=100.0, seed=5, size3d=((40, 40, 32), (64, 56, 40)),
                            size2d=((40, 60), (60, 90)), nt=(150, 200), freq=(20.0, 30.0))
    srv = SV.Server(max_bytes=4 << 30, chunk=8)
    try:
        stats = srv.run(reqs, fwi=fwi, t_limit=900.0)
    finally:
        srv.close()
    assert stats["done"] == len(reqs)
    plain = SV.FwiDriver(g, c0, w, shots, iterations=2, step0=step0)
    ctx = V.Context(0)
    try:
        mis_plain = plain.run_plain(ctx)
    finally:
        ctx.close()
    assert len(fwi.misfits) == len(mis_plain) >= 3
    assert fwi.misfits == mis_plain
    assert fwi.misfits[-1] < fwi.misfits[0]
