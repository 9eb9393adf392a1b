"""Golden cases: seeded inputs shared by make_golden.py (which runs the
reference binaries built by oracle/build_ref.sh) and the tests (which
regenerate the same inputs and compare against the stored outputs).

Inputs are regenerated, not stored; each fixture keeps a checksum of its
inputs so a change of generator is detected instead of silently compared.
"""
from __future__ import annotations

import hashlib
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "thesis-source-code_b200"))

import vtib200 as V  # noqa: E402
import vtib200.synth as S  # noqa: E402

GOLDEN = Path(__file__).resolve().parent


def digest(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()[:16]


def case3d(name: str) -> dict:
    """3D inputs: survey (starting model), observed data source model, boundaries."""
    if name == "g3_a":
        # nt = 64*2+2: the reference pipeline runs every level; 3-step sampling
        s = S.small3d(nx=40, ny=36, nz=32, nt=130, npad=8, rec_step=3, nshot=1, rate=2.1e-3)
    elif name == "g3_b":
        # nt not of the form 64k+2 (pipeline truncation), two shots, 4-step sampling
        s = S.small3d(nx=36, ny=40, nz=28, nt=100, npad=6, rec_step=4, nshot=2, seed=5,
                      rate=2.8e-3)
    elif name == "g3_c":
        # 2-step sampling: the reference's bookkeeping records only sample 1;
        # the source sits 2 cells under a receiver so that sample is non-zero
        s = S.survey3d(nx=36, ny=36, nz=32, nt=130, npad=8, d=10.0, dt=7e-4, rate=1.4e-3,
                       freq=25.0, rec_step=3, rec_start=4, rec_depth=30.0, src_depth=50.0,
                       seed=3, corr=30.0, src_xy=(19, 19))
    else:
        raise KeyError(name)
    true = S.small3d(nx=s.nx, ny=s.ny, nz=s.nz, nt=s.nt, npad=s.npad, seed=11)
    padb, randb = S.boundaries3d(s)
    return {"s": s, "cij": s.cij(), "cij_true": true.cij(), "padb": padb, "randb": randb,
            "shotid": np.arange(s.souloc.size // 5, dtype=np.int32)}


def case2d(name: str) -> dict:
    """2D survey (starting model), a true model for observed data, and a
    smooth model perturbation dc for the Gauss-Newton product."""
    if name == "g2_a":
        s = S.survey2d(nx=64, nz=40, nt=300, npad=10, d=10.0, dt=1e-3, rate=2e-3, freq=20.0,
                       src_x=300.0, src_z=50.0, rec_z=20.0, ns=2)
    else:
        raise KeyError(name)
    nnx, nnz = s.nx + 2 * s.npad, s.nz + 2 * s.npad
    rng = np.random.default_rng(21)
    bump = S.smooth(rng.standard_normal((nnz, nnx)).astype(np.float32), 4.0).reshape(-1)
    bump *= 0.05 / np.abs(bump).max()
    true = {k: (getattr(s, k) * (1 + bump)).astype(np.float32) for k in ("c11", "c13", "c33")}
    dc = {k: (getattr(s, k) * bump).astype(np.float32) for k in ("c11", "c13", "c33")}
    return {"s": s, "true": true, "dc": dc}


CASES3D = ["g3_a", "g3_b", "g3_c"]
# g3_c pins the recording bookkeeping only: with one recorded sample its
# gradient is ~1e-35, at the FP32 underflow limit, and not a meaningful check.
GRAD_CASES3D = ["g3_a", "g3_b"]
CASES2D = ["g2_a"]
# RTM fixtures (<case>_rtm.npz): the case's observed traces migrated with its
# starting model; in 3D the model carries the random boundary, as the RTM
# drivers pass it (rtm3d_f.cu:139-148).
RTM_CASES3D = ["g3_a"]
RTM_CASES2D = ["g2_a"]
# wavelet-gradient fixtures (<case>_wgrad.npz): the adjoint driven by the
# case's observed traces; in 3D the model carries the pad boundary (the
# sponge model), as the source-inversion drivers pass it.
WGRAD_CASES3D = ["g3_a"]
# gradient misfit options (<case>_misfit.npz), as the reference's tpow=,
# objtype=, halfwidth= parameters
MISFIT_CASES3D = ["g3_a"]
MISFIT_OPTIONS = {"agc": {"objtype": 1, "halfwidth": 8}, "tpow": {"tpow": 2.0}}
WGRAD_CASES2D = ["g2_a"]
# offset-domain image gathers (<case>_odcig.npz): half width in x offsets
ODCIG_CASES2D = {"g2_a": 6}


def pad_model3d(c: dict) -> np.ndarray:
    """cij of a 3D case with its pad boundary put into the pad region."""
    import vtib200 as V
    s = c["s"]
    n = s.nxyz
    return np.concatenate([V.put_boundary(c["padb"][k * s.nb:(k + 1) * s.nb],
                                          c["cij"][k * n:(k + 1) * n], s.nx, s.ny, s.nz,
                                          s.npad) for k in range(3)])


def rtm_model3d(c: dict) -> np.ndarray:
    """cij of a 3D case with its random boundary put into the pad region."""
    import vtib200 as V
    s = c["s"]
    n = s.nxyz
    return np.concatenate([V.put_boundary(c["randb"][k * s.nb:(k + 1) * s.nb],
                                          c["cij"][k * n:(k + 1) * n], s.nx, s.ny, s.nz,
                                          s.npad) for k in range(3)])


# Random-boundary generator cases: (n1, n2, n3, pad, pctG, seed); n3 = 1 is 2D.
RANDB_CASES = {"rb3_a": (40, 36, 30, 8, 0.9, 2017), "rb3_b": (48, 40, 36, 10, 0.6, 77),
               "rb2_a": (120, 80, 1, 20, 0.99, 5)}


def randb_input(name: str) -> np.ndarray:
    """Seeded velocity field of a random-boundary case."""
    n1, n2, n3, pad, pct, seed = RANDB_CASES[name]
    rng = np.random.default_rng(1234 + n1 + n3)
    return (1500 + 3000 * rng.random(n1 * n2 * n3)).astype(np.float32)
