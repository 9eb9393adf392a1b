"""Self-checks of the adjoint-state gradient in EXACT mode (FP64 oracle).

The reference's 3D gradient (objFuncGradient3d_f.cu:361-1111) propagates the
adjoint with the forward operator C.L, rebuilds the source field through a
random boundary and injects time-interpolated residuals, so it is not the
derivative of its own misfit and cannot pass a dot-product test. EXACT mode
fixes one discrete forward operator (plain diagonal sponge, every level,
receivers at their own cells) and its exact discrete adjoint (L.C form,
adjointCij of laplacian3d.ispc:166-190). These tests check:
  * the dot-product test <B dc, y> = <dc, B^T y> to 1e-6 (B: Born operator);
  * the Born operator against centred differences of the forward traces;
  * the gradient against centred finite differences of the misfit, sign
    included, with second-order convergence in the step.
"""
import numpy as np
import pytest

import oracle as O

import vtib200.synth as S

DOT_TOL = 1e-6
FD_TOL = 1e-4


@pytest.fixture(scope="module")
def case():
    s = S.small3d(nx=36, ny=32, nz=28, nt=120, npad=6, rec_step=3)
    true = S.small3d(nx=36, ny=32, nz=28, nt=120, npad=6, seed=11)
    n = s.nxyz
    c = s.cij().astype(np.float64)
    rng = np.random.default_rng(5)
    # perturbation with the model's own scale, zero nowhere
    dc = rng.standard_normal(3 * n) * c * 1e-2
    return dict(s=s, g=s.geom(), n=n, c=c, ct=true.cij().astype(np.float64), dc=dc, rng=rng)


def _split(c, n):
    return [c[k * n:(k + 1) * n] for k in range(3)]


def _fwd(k, c):
    s = k["s"]
    return O.exact_forward3d(k["g"], *_split(c, k["n"]), s.wavelet, s.souloc, [0], s.recloc)


def test_exact_dot_product(case):
    k, s = case, case["s"]
    d = _fwd(k, k["c"])
    assert np.abs(d).max() > 0
    y = k["rng"].standard_normal(d.size) * (d != 0)
    bd = O.exact_born3d(k["g"], *_split(k["c"], k["n"]), s.wavelet, s.souloc, [0], s.recloc,
                        k["dc"])
    bt = O.exact_adjoint3d(k["g"], *_split(k["c"], k["n"]), s.wavelet, s.souloc, [0], s.recloc, y)
    lhs, rhs = float(bd @ y), float(k["dc"] @ bt)
    assert lhs != 0.0
    assert abs(lhs - rhs) / abs(lhs) < DOT_TOL


def test_exact_born_matches_centred_difference_of_traces(case):
    k, s = case, case["s"]
    h = 1e-3
    fd = (_fwd(k, k["c"] + h * k["dc"]) - _fwd(k, k["c"] - h * k["dc"])) / (2 * h)
    bd = O.exact_born3d(k["g"], *_split(k["c"], k["n"]), s.wavelet, s.souloc, [0], s.recloc,
                        k["dc"])
    assert np.abs(bd).max() > 0
    assert np.linalg.norm(bd - fd) / np.linalg.norm(fd) < FD_TOL


def test_exact_gradient_matches_centred_fd_of_misfit(case):
    k, s = case, case["s"]
    dobs = _fwd(k, k["ct"])

    def misfit(c):
        r = _fwd(k, c) - dobs
        return 0.5 * float(r @ r), r

    j0, r0 = misfit(k["c"])
    assert j0 > 0
    grad = O.exact_adjoint3d(k["g"], *_split(k["c"], k["n"]), s.wavelet, s.souloc, [0],
                             s.recloc, r0)
    gdc = float(grad @ k["dc"])
    errs = []
    for h in (1e-2, 1e-3):
        fd = (misfit(k["c"] + h * k["dc"])[0] - misfit(k["c"] - h * k["dc"])[0]) / (2 * h)
        assert np.sign(fd) == np.sign(gdc)
        errs.append(abs(fd - gdc) / abs(fd))
    assert errs[1] < FD_TOL
    # centred differences converge at second order: 10x smaller step, ~100x smaller error
    assert errs[1] < errs[0] / 30
    # each model parameter's gradient on its own
    for p in range(3):
        dp = np.zeros_like(k["dc"])
        dp[p * k["n"]:(p + 1) * k["n"]] = k["dc"][p * k["n"]:(p + 1) * k["n"]]
        h = 1e-3
        fd = (misfit(k["c"] + h * dp)[0] - misfit(k["c"] - h * dp)[0]) / (2 * h)
        assert abs(fd - float(grad @ dp)) / abs(fd) < FD_TOL, p
