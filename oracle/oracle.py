"""ctypes loader for the CPU oracle (oracle/vti_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py, never by the library.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"
_lib = None
VP = C.c_void_p


def build():
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        for suf in ("f64", "f32"):
            f = getattr(L, f"orc3d_model_data_{suf}")
            f.argtypes = [VP] * 8 + [C.c_int, VP, VP, VP]
            f.restype = C.c_int
            f = getattr(L, f"orc3d_gradient_cij_{suf}")
            f.argtypes = [VP] * 8 + [C.c_int, VP, VP, VP, C.c_int, VP, C.c_float, C.c_int, C.c_int]
            f.restype = C.c_int
            f = getattr(L, f"orc3d_rtm_{suf}")
            f.argtypes = [VP] * 8 + [C.c_int, VP, VP, VP]
            f.restype = C.c_int
            f = getattr(L, f"orc2d_forward_{suf}")
            f.argtypes = [VP] * 7 + [C.c_int, VP, C.c_int, VP, VP, C.c_int]
            f.restype = C.c_int
        L.orc_max_threads.restype = C.c_int
        L.orc3d_damping.argtypes = [C.c_int] * 4 + [VP]
        L.orc3d_last_level.argtypes = [VP, VP]
        L.orc3d_last_level.restype = C.c_int
        for n in ("orc3d_time_forward_f32", "orc3d_time_backward_f32"):
            getattr(L, n).argtypes = [VP] * 5 + [C.c_int, VP]
            getattr(L, n).restype = C.c_int
        _lib = L
    return _lib


def _p(a):
    # data_as keeps a reference to the array, so a temporary made by _f32()
    # for this call lives until the call returns
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _geo3(g, full_steps=False, ref_gpus=1):
    ip = np.array([g.nx, g.ny, g.nz, g.nt, g.npad, 0 if full_steps else 1, ref_gpus],
                  dtype=np.int32)
    fp = np.array([g.ox, g.oy, g.oz, g.ot, g.dx, g.dy, g.dz, g.dt, g.sampling_rate],
                  dtype=np.float32)
    return ip, fp


def nnt3d(g):
    s = int(np.round(np.float32(g.sampling_rate) / np.float32(g.dt)))
    return (g.nt - 1) // s + 1


def model_data3d(g, c11, c13, c33, wavelet, souloc, shotid, recloc, dtype=np.float64,
                 full_steps=False, want_wavefield=False):
    """modelDataCij3d_f restated: traces (nnt*nrec_total) and optionally the
    last sigma_x level."""
    ip, fp = _geo3(g, full_steps)
    recloc = _f32(recloc).reshape(-1)
    out = np.zeros(nnt3d(g) * (recloc.size // 4), dtype=dtype)
    wf = np.zeros(g.nx * g.ny * g.nz, dtype=dtype) if want_wavefield else None
    suf = "f64" if dtype == np.float64 else "f32"
    shotid = _i32(shotid)
    getattr(lib(), f"orc3d_model_data_{suf}")(
        _p(ip), _p(fp), _p(_f32(c11)), _p(_f32(c13)), _p(_f32(c33)), _p(_f32(wavelet)),
        _p(_f32(souloc)), _p(shotid), len(shotid), _p(recloc), _p(out), _p(wf))
    return (out, wf) if want_wavefield else out


def gradient3d(g, cij, padb, randb, wavelet, souloc, shotid, recloc, dobs, dtype=np.float64,
               full_steps=False, misfit_only=False, want_modeled=False, tpow=0.0, objtype=0,
               halfwidth=20):
    """objFuncGradientCij3d_f restated: fgcij = [misfit/2, gc11, gc13, gc33];
    tpow / objtype / halfwidth as the reference's parameters of those names."""
    ip, fp = _geo3(g, full_steps)
    n = g.nx * g.ny * g.nz
    out = np.zeros(1 + 3 * n, dtype=dtype)
    recloc = _f32(recloc).reshape(-1)
    mod = np.zeros(nnt3d(g) * (recloc.size // 4), dtype=dtype) if want_modeled else None
    suf = "f64" if dtype == np.float64 else "f32"
    shotid = _i32(shotid)
    getattr(lib(), f"orc3d_gradient_cij_{suf}")(
        _p(ip), _p(fp), _p(_f32(cij)), _p(_f32(padb)), _p(_f32(randb)), _p(_f32(wavelet)),
        _p(_f32(souloc)), _p(shotid), len(shotid), _p(recloc), _p(_f32(dobs)), _p(out),
        1 if misfit_only else 0, _p(mod), tpow, objtype, halfwidth)
    return (out, mod) if want_modeled else out


def rtm3d(g, c11, c13, c33, wavelet, souloc, shotid, recloc, data, dtype=np.float64,
          full_steps=False):
    """rtmCij3d_f restated: the zero-lag image (nxyz), summed over shots."""
    ip, fp = _geo3(g, full_steps)
    out = np.zeros(g.nx * g.ny * g.nz, dtype=dtype)
    suf = "f64" if dtype == np.float64 else "f32"
    shotid = _i32(shotid)
    getattr(lib(), f"orc3d_rtm_{suf}")(
        _p(ip), _p(fp), _p(_f32(c11)), _p(_f32(c13)), _p(_f32(c33)), _p(_f32(wavelet)),
        _p(_f32(souloc)), _p(shotid), len(shotid), _p(_f32(recloc).reshape(-1)), _p(_f32(data)),
        _p(out))
    return out


def odcig3d(g, c11, c13, c33, wavelet, souloc, shotid, recloc, data, nlag, dtype=np.float64,
            full_steps=False):
    """Offset-domain gathers of rtmCij3d_f's migration with the extended
    imaging condition of extendedImagingKernel (wave3d.cu:1299-1313):
    (2 nlag + 1) x nxyz, lag -nlag first."""
    ip, fp = _geo3(g, full_steps)
    n = g.nx * g.ny * g.nz
    out = np.zeros((2 * nlag + 1) * n, dtype=dtype)
    suf = "f64" if dtype == np.float64 else "f32"
    f = getattr(lib(), f"orc3d_odcig_{suf}")
    f.argtypes = [VP] * 8 + [C.c_int, VP, VP, C.c_int, VP]
    f.restype = C.c_int
    shotid = _i32(shotid)
    st = f(_p(ip), _p(fp), _p(_f32(c11)), _p(_f32(c13)), _p(_f32(c33)), _p(_f32(wavelet)),
           _p(_f32(souloc)), _p(shotid), len(shotid), _p(_f32(recloc).reshape(-1)),
           _p(_f32(data)), int(nlag), _p(out))
    assert st == 0
    return out.reshape(2 * nlag + 1, n)


def wavelet_gradient3d(g, c11, c13, c33, souloc, shotid, recloc, data, dtype=np.float64,
                       full_steps=False):
    """waveletGradientCij3d_f restated: the gradient w.r.t. the wavelet (nt)."""
    ip, fp = _geo3(g, full_steps)
    out = np.zeros(g.nt, dtype=dtype)
    suf = "f64" if dtype == np.float64 else "f32"
    f = getattr(lib(), f"orc3d_wavelet_gradient_{suf}")
    f.argtypes = [VP] * 7 + [C.c_int, VP, VP, VP]
    f.restype = C.c_int
    shotid = _i32(shotid)
    f(_p(ip), _p(fp), _p(_f32(c11)), _p(_f32(c13)), _p(_f32(c33)), _p(_f32(souloc)), _p(shotid),
      len(shotid), _p(_f32(recloc).reshape(-1)), _p(_f32(data)), _p(out))
    return out


def _exact3d(name, g, c11, c13, c33, wavelet, souloc, shotid, recloc, extra, n_out):
    ip, fp = _geo3(g, full_steps=True)
    f = getattr(lib(), name)
    f.argtypes = [VP] * 8 + [C.c_int] + [VP] * (2 + len(extra))
    f.restype = C.c_int
    out = np.zeros(n_out)
    shotid = _i32(shotid)
    f(_p(ip), _p(fp), *[_p(np.ascontiguousarray(a, dtype=np.float64)) for a in (c11, c13, c33)],
      _p(_f32(wavelet)), _p(_f32(souloc)), _p(shotid), len(shotid), _p(_f32(recloc).reshape(-1)),
      *[_p(np.ascontiguousarray(e, dtype=np.float64)) for e in extra], _p(out))
    return out


def exact_forward3d(g, c11, c13, c33, wavelet, souloc, shotid, recloc):
    """EXACT-mode traces (self-check operator, every level up to nt-1); the
    model is taken in FP64."""
    nrec = np.asarray(recloc).size // 4
    return _exact3d("orc3d_exact_forward", g, c11, c13, c33, wavelet, souloc, shotid, recloc,
                    [], nnt3d(g) * nrec)


def exact_born3d(g, c11, c13, c33, wavelet, souloc, shotid, recloc, dc):
    """Derivative of the EXACT traces along dc = (dc11, dc13, dc33) stacked."""
    nrec = np.asarray(recloc).size // 4
    return _exact3d("orc3d_exact_born", g, c11, c13, c33, wavelet, souloc, shotid, recloc,
                    [dc], nnt3d(g) * nrec)


def exact_adjoint3d(g, c11, c13, c33, wavelet, souloc, shotid, recloc, res):
    """Transpose of exact_born3d applied to traces res: with res = modeled -
    observed, the gradient (dJ/dc11, dJ/dc13, dJ/dc33 stacked) of
    J = 1/2 |modeled - observed|^2."""
    return _exact3d("orc3d_exact_adjoint", g, c11, c13, c33, wavelet, souloc, shotid, recloc,
                    [res], 3 * g.nx * g.ny * g.nz)


def exact_gnhv3d(g, c11, c13, c33, wavelet, souloc, shotid, recloc, dc):
    """H dc = B^T B dc in EXACT mode (B: Born operator), FP64."""
    bd = exact_born3d(g, c11, c13, c33, wavelet, souloc, shotid, recloc, dc)
    return exact_adjoint3d(g, c11, c13, c33, wavelet, souloc, shotid, recloc, bd)


# ------------------------------------------------------------ host glue
# numpy restatements of the reference's host helpers, so that inputs can be
# built with the oracle alone (the reference leg of the benchmark)
def _pad_mask(nx, ny, nz, npad):
    m = np.ones((nz, ny, nx), dtype=bool)
    m[npad:nz - npad, npad:ny - npad, npad:nx - npad] = False
    return m


def get_boundary(v, nx, ny, nz, npad):
    """getBoundary (lib/vti-fwi-3d/gpu/boundary.cpp:10-46): the pad-region
    cells in index order (top planes, then per middle plane the npad full
    rows, both npad-wide ends of each middle row, the npad full rows, then
    the bottom planes): the cells of the pad mask in raster order."""
    return _f32(v).reshape(nz, ny, nx)[_pad_mask(nx, ny, nz, npad)].copy()


def put_boundary(b, v, nx, ny, nz, npad):
    """putBoundary (boundary.cpp:48-84): the inverse of get_boundary."""
    out = np.array(v, dtype=np.float32, copy=True).reshape(nz, ny, nx)
    out[_pad_mask(nx, ny, nz, npad)] = _f32(b)
    return out.reshape(-1)


def vepsdel_to_cij(v, eps, dl, v0=1.0, eps0=1.0, del0=1.0):
    """VEpsDel2Cij (lib/vti-fwi-2d/conversions.cpp:42-50) with its float /
    double mix: c33 = v0 v0 v v in float; c11 = c33 (1. + 2 eps0 eps) and
    c13 = c33 sqrt(1. + 2 del0 del) in double, stored as float."""
    f = np.float32
    v, eps, dl = _f32(v), _f32(eps), _f32(dl)
    c33 = (f(v0) * f(v0) * v * v).astype(np.float32)
    te = 1.0 + ((f(2) * f(eps0)) * eps).astype(np.float64)
    td = np.sqrt(1.0 + ((f(2) * f(del0)) * dl).astype(np.float64))
    c11 = (c33.astype(np.float64) * te).astype(np.float32)
    c13 = (c33.astype(np.float64) * td).astype(np.float32)
    return c11, c13, c33


def damping3d(nx, ny, nz, npad):
    out = np.zeros(nx * ny + nz, dtype=np.float32)
    lib().orc3d_damping(nx, ny, nz, npad, _p(out))
    return out[: nx * ny].reshape(ny, nx), out[nx * ny:]


def last_level(g, full_steps=False):
    ip, fp = _geo3(g, full_steps)
    return lib().orc3d_last_level(_p(ip), _p(fp))


def forward2d(g, c11, c13, c33, wavelet, sloc, rloc, taper, mode=0, slocxz=None,
              dtype=np.float64):
    """mode 0: synthetic_f traces [rows, nr]; mode 1: modeling_f snapshots."""
    ip = np.array([g.nx, g.nz, g.nt, g.npad], dtype=np.int32)
    fp = np.array([g.dx, g.dz, g.dt, g.rate, g.ot], dtype=np.float32)
    nnxz = (g.nx + 2 * g.npad) * (g.nz + 2 * g.npad)
    suf = "f64" if dtype == np.float64 else "f32"
    if mode == 0:
        sloc, rloc = _i32(sloc).reshape(-1), _i32(rloc).reshape(-1)
        nr = rloc.size // 2
        ratio = int(np.float32(g.rate) / np.float32(g.dt) + np.float32(0.5))
        nt_neg = int(round(abs(g.ot) / g.dt))
        rows = (g.nt - nt_neg - 1) // ratio + 1
        out = np.zeros(rows * nr, dtype=dtype)
        getattr(lib(), f"orc2d_forward_{suf}")(
            _p(ip), _p(fp), _p(_f32(c11)), _p(_f32(c13)), _p(_f32(c33)), _p(_f32(wavelet)),
            _p(sloc), sloc.size // 4, _p(rloc), nr, _p(_f32(taper)), _p(out), 0)
        return out.reshape(rows, nr)
    ratio = int(np.round(np.float32(g.rate) / np.float32(g.dt)))
    nt_neg = int(round(abs(g.ot) / g.dt))
    rows = max((g.nt - 1 - nt_neg) // ratio + 1, 2)
    out = np.zeros(rows * nnxz, dtype=dtype)
    s = np.array([slocxz], dtype=np.int32)
    getattr(lib(), f"orc2d_forward_{suf}")(
        _p(ip), _p(fp), _p(_f32(c11)), _p(_f32(c13)), _p(_f32(c33)), _p(_f32(wavelet)), _p(s), 1,
        None, 0, _p(_f32(taper)), _p(out), 1)
    return out.reshape(rows, nnxz)


def max_threads():
    """OpenMP threads of the oracle's parallel loops."""
    return lib().orc_max_threads()


def time_forward_f32(g, c11, c13, c33, nsteps):
    """Runs nsteps FP32 forward steps; returns threads used."""
    ip, fp = _geo3(g)
    n = g.nx * g.ny * g.nz
    scratch = np.zeros(4 * n, dtype=np.float32)
    return lib().orc3d_time_forward_f32(_p(ip), _p(fp), _p(_f32(c11)), _p(_f32(c13)),
                                        _p(_f32(c33)), nsteps, _p(scratch))


def time_backward_f32(g, c11, c13, c33, nsteps):
    ip, fp = _geo3(g)
    n = g.nx * g.ny * g.nz
    scratch = np.zeros(11 * n, dtype=np.float32)
    return lib().orc3d_time_backward_f32(_p(ip), _p(fp), _p(_f32(c11)), _p(_f32(c13)),
                                         _p(_f32(c33)), nsteps, _p(scratch))


def rtm2d(g, c11, c13, c33, wavelet, sloc, rloc, taper, data, dtype=np.float64):
    """rtm_f restated: the image (nnxz), summed over shots."""
    suf = "f64" if dtype == np.float64 else "f32"
    f = getattr(lib(), f"orc2d_rtm_{suf}")
    f.argtypes = [VP] * 8 + [C.c_int, VP, C.c_int, VP, VP]
    f.restype = C.c_int
    ip = np.array([g.nx, g.nz, g.nt, g.npad], dtype=np.int32)
    fp = np.array([g.dx, g.dz, g.dt, g.rate, g.ot], dtype=np.float32)
    out = np.zeros((g.nx + 2 * g.npad) * (g.nz + 2 * g.npad), dtype=dtype)
    sloc, rloc = _i32(sloc).reshape(-1), _i32(rloc).reshape(-1)
    f(_p(ip), _p(fp), _p(_f32(c11)), _p(_f32(c13)), _p(_f32(c33)), _p(_f32(wavelet)),
      _p(_f32(data)), _p(sloc), sloc.size // 4, _p(rloc), rloc.size // 2, _p(_f32(taper)),
      _p(out))
    return out


def odcig2d(g, nhx, c11, c13, c33, wavelet, sloc, rloc, taper, data, dtype=np.float64):
    """odcig_f restated: offset-domain image gathers, (2 nhx + 1) x nnxz."""
    suf = "f64" if dtype == np.float64 else "f32"
    f = getattr(lib(), f"orc2d_odcig_{suf}")
    f.argtypes = [VP, VP, C.c_int] + [VP] * 6 + [C.c_int, VP, C.c_int, VP, VP]
    f.restype = C.c_int
    ip = np.array([g.nx, g.nz, g.nt, g.npad], dtype=np.int32)
    fp = np.array([g.dx, g.dz, g.dt, g.rate, g.ot], dtype=np.float32)
    nnxz = (g.nx + 2 * g.npad) * (g.nz + 2 * g.npad)
    out = np.zeros((2 * nhx + 1) * nnxz, dtype=dtype)
    sloc, rloc = _i32(sloc).reshape(-1), _i32(rloc).reshape(-1)
    f(_p(ip), _p(fp), nhx, _p(_f32(c11)), _p(_f32(c13)), _p(_f32(c33)), _p(_f32(wavelet)),
      _p(_f32(data)), _p(sloc), sloc.size // 4, _p(rloc), rloc.size // 2, _p(_f32(taper)),
      _p(out))
    return out.reshape(2 * nhx + 1, nnxz)


def wavelet_gradient2d(g, c11, c13, c33, sloc, rloc, taper, data, dtype=np.float64):
    """waveletGradient_f restated: the gradient w.r.t. the wavelet (nt)."""
    suf = "f64" if dtype == np.float64 else "f32"
    f = getattr(lib(), f"orc2d_wavelet_gradient_{suf}")
    f.argtypes = [VP] * 7 + [C.c_int, VP, C.c_int, VP, VP]
    f.restype = C.c_int
    ip = np.array([g.nx, g.nz, g.nt, g.npad], dtype=np.int32)
    fp = np.array([g.dx, g.dz, g.dt, g.rate, g.ot], dtype=np.float32)
    out = np.zeros(g.nt, dtype=dtype)
    sloc, rloc = _i32(sloc).reshape(-1), _i32(rloc).reshape(-1)
    f(_p(ip), _p(fp), _p(_f32(c11)), _p(_f32(c13)), _p(_f32(c33)), _p(_f32(data)), _p(sloc),
      sloc.size // 4, _p(rloc), rloc.size // 2, _p(_f32(taper)), _p(out))
    return out


def gradient2d(g, c11, c13, c33, wavelet, sloc, rloc, taper, data=None, dc=None,
               dtype=np.float64):
    """objFuncGradient_f (dc None) or GNhessian_f (dc = (dc11, dc13, dc33))
    restated; returns (gc11, gc13, gc33, misfit/2)."""
    L = lib()
    suf = "f64" if dtype == np.float64 else "f32"
    f = getattr(L, f"orc2d_gradient_{suf}")
    f.argtypes = [VP] * 10 + [C.c_int, VP, C.c_int, VP, VP, VP, VP, VP, C.c_int]
    f.restype = C.c_double
    ip = np.array([g.nx, g.nz, g.nt, g.npad], dtype=np.int32)
    fp = np.array([g.dx, g.dz, g.dt, g.rate, g.ot], dtype=np.float32)
    n = (g.nx + 2 * g.npad) * (g.nz + 2 * g.npad)
    out = [np.zeros(n, dtype=dtype) for _ in range(3)]
    sloc, rloc = _i32(sloc).reshape(-1), _i32(rloc).reshape(-1)
    born = dc is not None
    d11, d13, d33 = (None, None, None) if not born else tuple(_f32(x) for x in dc)
    dat = None if data is None else _f32(data)
    mis = f(_p(ip), _p(fp), _p(_f32(c11)), _p(_f32(c13)), _p(_f32(c33)), _p(d11), _p(d13),
            _p(d33), _p(_f32(wavelet)), _p(sloc), sloc.size // 4, _p(rloc), rloc.size // 2,
            _p(_f32(taper)), _p(dat), _p(out[0]), _p(out[1]), _p(out[2]), 1 if born else 0)
    return out[0], out[1], out[2], mis
