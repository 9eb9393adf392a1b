"""Seeded synthetic inputs for the VTI path (no datasets exist for it).

Models, wavelets and acquisition geometry follow the workloads the path is
benchmarked on: a 5-layer VTI model (v 1500->4500 m/s, eps 0->0.2,
delta 0->0.1) with a -10% Gaussian velocity anomaly, a Ricker source and a
surface receiver line (2D) or grid (3D). All arrays are float32 in the
reference layouts (3D x-fastest with the pad inside n; 2D (nx+2npad) x
(nz+2npad)).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
from scipy.ndimage import uniform_filter


def smooth(a, sigma_cells, mode="nearest"):
    """Gaussian-like smoothing by three box-filter passes per axis (variance
    3(w^2-1)/12 = sigma^2); O(n) per pass whatever the width."""
    a = np.asarray(a, dtype=np.float32)
    if sigma_cells <= 0:
        return a.copy()
    w = max(1, int(round(np.sqrt(4.0 * sigma_cells**2 + 1.0))))
    for _ in range(3):
        a = uniform_filter(a, size=w, mode=mode)
    return a.astype(np.float32)

V_LAYERS = np.array([1500.0, 2250.0, 3000.0, 3750.0, 4500.0], dtype=np.float32)
EPS_LAYERS = np.array([0.0, 0.05, 0.10, 0.15, 0.20], dtype=np.float32)
DEL_LAYERS = np.array([0.0, 0.025, 0.05, 0.075, 0.10], dtype=np.float32)


def ricker(nt, dt, freq, ot=0.0, tdelay=None, scale=1.0):
    """Ricker wavelet with the float arithmetic of lib/vti-fwi-2d/ricker.cpp:11-21."""
    if tdelay is None:
        tdelay = 1.2 / freq
    pi = np.float64(4.0 * np.arctan(1.0))
    pi2f2 = np.float32(pi * pi * freq * freq)
    it = np.arange(nt)
    t = (it * np.float32(dt) + np.float32(ot) - np.float32(tdelay)).astype(np.float32)
    a = (pi2f2 * t * t).astype(np.float32)
    w = ((1.0 - 2.0 * a.astype(np.float64)) * np.exp(-a.astype(np.float64))).astype(np.float32)
    return (w * np.float32(scale)).astype(np.float32)


def _layer_index(depth, interfaces):
    return np.searchsorted(interfaces, depth, side="right")


def layered(depth, interfaces):
    """v, eps, del of the 5-layer model at the given depths (m)."""
    k = _layer_index(depth, interfaces)
    return V_LAYERS[k], EPS_LAYERS[k], DEL_LAYERS[k]


def interfaces_for(depth_max, seed=1, lo_frac=0.1, hi_frac=0.9):
    rng = np.random.default_rng(seed)
    return np.sort(rng.uniform(lo_frac * depth_max, hi_frac * depth_max, size=4))


@dataclass
class Survey3d:
    nx: int
    ny: int
    nz: int
    nt: int
    npad: int
    d: float
    dt: float
    rate: float
    o: float
    v: np.ndarray
    eps: np.ndarray
    dl: np.ndarray
    wavelet: np.ndarray
    souloc: np.ndarray
    recloc: np.ndarray
    extra: dict = field(default_factory=dict)

    @property
    def nxyz(self):
        return self.nx * self.ny * self.nz

    def geom(self):
        from . import geom3d
        return geom3d(self.nx, self.ny, self.nz, self.nt, self.npad, self.d, self.d, self.d,
                      self.dt, self.rate, ox=self.o, oy=self.o, oz=self.o, ot=0.0)

    def cij(self, v=None, eps=None, dl=None):
        from . import vepsdel_to_cij
        v = self.v if v is None else v
        eps = self.eps if eps is None else eps
        dl = self.dl if dl is None else dl
        c11, c13, c33 = vepsdel_to_cij(v, eps, dl)
        return np.concatenate([c11, c13, c33])

    @property
    def nb(self):
        n, p = (self.nx, self.ny, self.nz), self.npad
        return n[0] * n[1] * n[2] - (n[0] - 2 * p) * (n[1] - 2 * p) * (n[2] - 2 * p)


def grf(shape, corr_cells, std, clip, seed):
    """Gaussian random field: smoothed white noise scaled to `std`, clipped."""
    rng = np.random.default_rng(seed)
    f = smooth(rng.standard_normal(shape).astype(np.float32), corr_cells, mode="wrap")
    f *= std / max(f.std(), 1e-30)
    return np.clip(f, -clip, clip).astype(np.float32)


def random_boundary(v, nx, ny, nz, npad, seed, lo=0.7):
    """Random-boundary velocity: v times a seeded multiplier in [lo, 1) inside
    the pad, smoothly growing in strength with the distance into the pad.
    The multiplier is <= 1 so the random pass stays within the CFL bound of
    the model (the reference generator also only lowers velocity,
    lib/random-boundary/randomBound.h:233-248)."""
    rng = np.random.default_rng(seed)
    vv = v.reshape(nz, ny, nx).astype(np.float32).copy()

    def depth(n):
        i = np.arange(n)
        return np.maximum(np.maximum(npad - i, i - (n - 1 - npad)), 0).astype(np.float32)

    dist = np.maximum(np.maximum(depth(nx)[None, None, :], depth(ny)[None, :, None]),
                      depth(nz)[:, None, None])
    pct = np.clip(dist / max(npad, 1), 0, 1)
    r = 1.0 - pct * (1.0 - lo) * rng.uniform(0.0, 1.0, size=vv.shape).astype(np.float32)
    vv = np.where(dist > 0, vv * r, vv)
    return vv.reshape(-1).astype(np.float32)


def survey3d(nx=400, ny=400, nz=200, nt=3010, npad=40, d=12.5, dt=1e-3, rate=4e-3, freq=12.0,
             rec_step=2, rec_depth=25.0, src_depth=25.0, seed=3, grf_std=0.05, grf_clip=0.10,
             corr=200.0, smooth_m=None, rec_start=4, src_xy=None):
    """3D layered VTI survey (one shot at the centre, receiver grid at depth).

    The physical origin is the first interior cell (o = -npad*d), so depths
    are measured from the top of the interior. With smooth=<metres> the
    returned model is the true model smoothed by a Gaussian of that width
    (the starting model of an inversion); the true model is in extra['true'].
    """
    o = -npad * d
    z = (np.arange(nz) * d + o).astype(np.float32)
    zi = np.clip(z, 0, None)
    interior_depth = (nz - 2 * npad) * d
    inter = interfaces_for(interior_depth, seed=1)
    v1, e1, d1 = layered(zi, inter)
    shape = (nz, ny, nx)
    v = np.broadcast_to(v1[:, None, None], shape).astype(np.float32).copy()
    eps = np.broadcast_to(e1[:, None, None], shape).astype(np.float32).copy()
    dl = np.broadcast_to(d1[:, None, None], shape).astype(np.float32).copy()
    # -10% Gaussian velocity anomaly at the centre of the interior
    xs = (np.arange(nx) * d + o)[None, None, :]
    ys = (np.arange(ny) * d + o)[None, :, None]
    zs = z[:, None, None]
    cx, cy, cz = (nx - 2 * npad) * d / 2, (ny - 2 * npad) * d / 2, interior_depth * 0.6
    sig = 150.0 if interior_depth > 600 else interior_depth / 6
    v *= (1.0 - 0.1 * np.exp(-((xs - cx) ** 2 + (ys - cy) ** 2 + (zs - cz) ** 2) / (2 * sig**2))
          ).astype(np.float32)
    if grf_std > 0:
        cc = corr / d
        v *= 1 + grf(shape, cc, grf_std, grf_clip, seed)
        eps *= 1 + grf(shape, cc, grf_std, grf_clip, seed + 100)
        dl *= 1 + grf(shape, cc, grf_std, grf_clip, seed + 200)
        dl = np.minimum(dl, eps)
    true = (v.reshape(-1).copy(), eps.reshape(-1).copy(), dl.reshape(-1).copy())
    if smooth_m:
        s = smooth_m / d
        v, eps, dl = smooth(v, s), smooth(eps, s), smooth(dl, s)
    wavelet = ricker(nt, dt, freq)
    # receivers on every rec_step-th cell of the update region
    rx = np.arange(rec_start, nx - rec_start, rec_step)
    ry = np.arange(rec_start, ny - rec_start, rec_step)
    RX, RY = np.meshgrid(rx, ry, indexing="xy")
    nr = RX.size
    recloc = np.zeros((nr, 4), dtype=np.float32)
    recloc[:, 0] = RX.reshape(-1) * d + o + 0.25 * d
    recloc[:, 1] = RY.reshape(-1) * d + o + 0.25 * d
    recloc[:, 2] = rec_depth + 0.25 * d
    recloc[:, 3] = 1.0
    sx, sy = (nx // 2, ny // 2) if src_xy is None else src_xy
    souloc = np.array([[sx * d + o + 0.25 * d, sy * d + o + 0.25 * d,
                        src_depth + 0.25 * d, nr, 0]], dtype=np.float32)
    return Survey3d(nx, ny, nz, nt, npad, d, dt, rate, o, v.reshape(-1).astype(np.float32),
                    eps.reshape(-1).astype(np.float32), dl.reshape(-1).astype(np.float32),
                    wavelet, souloc.reshape(-1), recloc.reshape(-1), extra={"true": true})


# The headline gradient workload: a 400 x 400 x 200 grid at 12.5 m with a
# 40-cell pad inside it, dt 1 ms, nt 3000, 12 Hz Ricker, a 200 x 200 receiver
# grid at 25 m spacing and 25 m depth, 4 ms trace sampling, gradient at the
# true model smoothed by a 250 m Gaussian.
GRADIENT400 = dict(nx=400, ny=400, nz=200, nt=3000, npad=40, d=12.5, dt=1e-3, rate=4e-3,
                   freq=12.0, rec_step=2, rec_start=0, rec_depth=25.0, src_depth=25.0,
                   smooth_m=250.0)


def gradient_inputs(kw, rank=0, get_boundary=None, put_boundary=None, vepsdel_to_cij=None):
    """Inputs of one shot of a gradient workload (kwargs of survey3d): the
    survey, the starting c_ij, the true c_ij with the pad boundary of the true
    model (what observed data are modeled with), and the pad and random
    boundary lists. Each rank's shot sits at its own offset from the centre.
    The three host functions default to the library's; any implementation of
    boundary.cpp:10-46 and conversions.cpp:42-50 gives the same arrays."""
    if get_boundary is None or put_boundary is None or vepsdel_to_cij is None:
        from . import get_boundary as gb, put_boundary as pb, vepsdel_to_cij as vc
        get_boundary, put_boundary, vepsdel_to_cij = (get_boundary or gb, put_boundary or pb,
                                                      vepsdel_to_cij or vc)
    kw = dict(kw)
    nx, ny = kw["nx"], kw["ny"]
    off = [(0, 0), (40, 0), (0, 40), (40, 40), (-40, 0), (0, -40), (-40, -40), (40, -40)]
    dx, dy = off[rank % len(off)]
    kw["src_xy"] = (nx // 2 + dx * nx // 400, ny // 2 + dy * ny // 400)
    s = survey3d(**kw)
    padb, randb = boundaries3d(s, get_boundary=get_boundary, vepsdel_to_cij=vepsdel_to_cij)
    n = s.nxyz
    cstart = np.concatenate(vepsdel_to_cij(s.v, s.eps, s.dl))
    ctrue = np.concatenate(vepsdel_to_cij(*s.extra["true"]))
    ctrue = np.concatenate([put_boundary(padb[k * s.nb:(k + 1) * s.nb], ctrue[k * n:(k + 1) * n],
                                         s.nx, s.ny, s.nz, s.npad) for k in range(3)])
    return s, cstart.astype(np.float32), ctrue.astype(np.float32), padb, randb


def small3d(nx=48, ny=44, nz=40, nt=130, npad=8, d=10.0, dt=7e-4, rate=1.4e-3, freq=25.0,
            seed=3, rec_step=3, nshot=1):
    """A reduced 3D survey for parity tests (CFL-safe: dt^2 lambda_max < 4)."""
    s = survey3d(nx=nx, ny=ny, nz=nz, nt=nt, npad=npad, d=d, dt=dt, rate=rate, freq=freq,
                 rec_step=rec_step, rec_depth=3 * d, src_depth=5 * d, seed=seed,
                 corr=3 * d, smooth_m=None)
    if nshot > 1:
        rng = np.random.default_rng(seed + 7)
        nr = s.recloc.size // 4
        so = []
        for k in range(nshot):
            ix = int(rng.integers(npad, nx - npad))
            iy = int(rng.integers(npad, ny - npad))
            so.append([ix * d + s.o + 0.25 * d, iy * d + s.o + 0.25 * d, 5 * d + 0.25 * d,
                       nr, 0])
        s.souloc = np.array(so, dtype=np.float32).reshape(-1)
    return s


def boundaries3d(s: Survey3d, v_true=None, seed=4, get_boundary=None, vepsdel_to_cij=None):
    """pad and random boundary lists of c11,c13,c33 (3*nb floats each) built
    the way objFuncGradientVEpsDel does (objFuncGradient3d_f.cu:261-269).
    get_boundary / vepsdel_to_cij default to the library's host functions."""
    if get_boundary is None or vepsdel_to_cij is None:
        from . import get_boundary as gb, vepsdel_to_cij as vc
        get_boundary = get_boundary or gb
        vepsdel_to_cij = vepsdel_to_cij or vc
    v = s.v if v_true is None else v_true
    bv = get_boundary(v, s.nx, s.ny, s.nz, s.npad)
    be = get_boundary(s.eps, s.nx, s.ny, s.nz, s.npad)
    bd = get_boundary(s.dl, s.nx, s.ny, s.nz, s.npad)
    vr = random_boundary(v, s.nx, s.ny, s.nz, s.npad, seed)
    bvr = get_boundary(vr, s.nx, s.ny, s.nz, s.npad)
    padb = np.concatenate(vepsdel_to_cij(bv, be, bd))
    randb = np.concatenate(vepsdel_to_cij(bvr, be, bd))
    return padb, randb


@dataclass
class Survey2d:
    nx: int
    nz: int
    nt: int
    npad: int
    d: float
    dt: float
    rate: float
    c11: np.ndarray
    c13: np.ndarray
    c33: np.ndarray
    wavelet: np.ndarray
    sloc: np.ndarray
    rloc: np.ndarray
    taper: np.ndarray

    def geom(self):
        from . import geom2d
        return geom2d(self.nx, self.nz, self.nt, self.npad, self.d, self.d, self.dt, self.rate)


def survey2d(nx=401, nz=201, nt=2000, npad=30, d=10.0, dt=1e-3, rate=2e-3, freq=15.0,
             src_x=2000.0, src_z=20.0, rec_z=20.0, seed=1, ns=1):
    """2D layered VTI survey (lib/vti-fwi-2d conventions)."""
    from . import init_taper2d, vepsdel_to_cij
    nnx, nnz = nx + 2 * npad, nz + 2 * npad
    z = (np.arange(nnz) - npad) * d
    x = (np.arange(nnx) - npad) * d
    inter = interfaces_for((nz - 1) * d, seed=seed)
    v1, e1, d1 = layered(np.clip(z, 0, (nz - 1) * d), inter)
    v = np.broadcast_to(v1[:, None], (nnz, nnx)).astype(np.float32).copy()
    eps = np.broadcast_to(e1[:, None], (nnz, nnx)).astype(np.float32).copy()
    dl = np.broadcast_to(d1[:, None], (nnz, nnx)).astype(np.float32).copy()
    xc = min(2000.0, (nx - 1) * d / 2)
    zc = min(1000.0, (nz - 1) * d / 2)
    sig = min(150.0, (nz - 1) * d / 8)
    X, Z = np.meshgrid(np.clip(x, 0, (nx - 1) * d), np.clip(z, 0, (nz - 1) * d), indexing="xy")
    v *= (1 - 0.1 * np.exp(-((X - xc) ** 2 + (Z - zc) ** 2) / (2 * sig**2))).astype(np.float32)
    c11, c13, c33 = vepsdel_to_cij(v.reshape(-1), eps.reshape(-1), dl.reshape(-1))
    wavelet = ricker(nt, dt, freq)
    nr = nx
    rloc = np.zeros((nr, 2), dtype=np.int32)
    rloc[:, 0] = np.arange(nr) + npad
    rloc[:, 1] = int(rec_z / d + 0.5) + npad
    sx = [int(min(src_x, (nx - 1) * d) / d + 0.5) + npad]
    if ns > 1:
        sx = list(np.linspace(npad + 4, npad + nx - 5, ns).astype(int))
    sloc = np.array([[s, int(src_z / d + 0.5) + npad, nr, 0] for s in sx], dtype=np.int32)
    taper = init_taper2d(nx, nz, npad)
    return Survey2d(nx, nz, nt, npad, d, dt, rate, c11, c13, c33, wavelet, sloc.reshape(-1),
                    rloc.reshape(-1), taper)


def batch_windows(nx, ny, nshot, amin, amax, seed=5):
    """Per-shot windows (x0, y0, ax, ay) of a batched survey: apertures per
    side drawn uniformly from [amin, amax] (seeded, clipped to the model),
    window centres on a regular grid of shot positions over the model."""
    rng = np.random.default_rng(seed)
    g = int(np.ceil(np.sqrt(nshot)))
    wins = []
    for k in range(nshot):
        ax = int(min(rng.integers(amin, amax + 1), nx))
        ay = int(min(rng.integers(amin, amax + 1), ny))
        cx = int((k % g + 0.5) * nx / g)
        cy = int((k // g + 0.5) * ny / g)
        x0 = int(np.clip(cx - ax // 2, 0, nx - ax))
        y0 = int(np.clip(cy - ay // 2, 0, ny - ay))
        wins.append((x0, y0, ax, ay))
    return wins


def batch_survey3d(s: Survey3d, windows, rec_step=2, rec_depth=None, src_depth=None):
    """Sources and receivers of a batched survey on the model of s: one shot
    per window, the source at the window's centre cell, receivers on every
    rec_step-th cell of the window's interior (outside its npad frame).
    Returns (souloc: 5 floats per shot, recloc: 4 floats per receiver, one
    global list, each shot's receivers contiguous)."""
    d, o, npad = s.d, s.o, s.npad
    rz = (3 * d if rec_depth is None else rec_depth) + 0.25 * d
    sz = (5 * d if src_depth is None else src_depth) + 0.25 * d
    so, rec = [], []
    for (x0, y0, ax, ay) in windows:
        rx = np.arange(x0 + npad, x0 + ax - npad, rec_step)
        ry = np.arange(y0 + npad, y0 + ay - npad, rec_step)
        RX, RY = np.meshgrid(rx, ry, indexing="xy")
        first = sum(len(r) for r in rec)
        r = np.zeros((RX.size, 4), dtype=np.float32)
        r[:, 0] = RX.reshape(-1) * d + o + 0.25 * d
        r[:, 1] = RY.reshape(-1) * d + o + 0.25 * d
        r[:, 2] = rz
        r[:, 3] = 1.0
        rec.append(r)
        cx, cy = x0 + ax // 2, y0 + ay // 2
        so.append([cx * d + o + 0.25 * d, cy * d + o + 0.25 * d, sz, RX.size, first])
    return (np.array(so, dtype=np.float32).reshape(-1),
            np.concatenate(rec).astype(np.float32).reshape(-1))
