"""vti2d_synthetic_noalloc against vti2d_synthetic, through the C ABI.

The allocation-free entry point keeps all device data of a call in one static
device array; it must give the traces of the allocating entry point on the
same inputs, on consecutive calls (the array is reused, so whatever must start
at zero has to be cleared by each call), and must reject a call larger than
its array before doing any work. This file is collected last so the check
also runs after every other GPU test has used the device.
"""
import ctypes as C

import numpy as np
import pytest

import cases as K
from conftest import rel_l2

import vtib200 as V
import vtib200.synth as S

pytestmark = pytest.mark.gpu

TRACE_TOL = 1e-5  # FP32 trace tolerance of the 2D parity tests


def _traces(ctx, name, g, s):
    sloc = V._i32(s.sloc).reshape(-1)
    rloc = V._i32(s.rloc).reshape(-1)
    nr = rloc.size // 2
    ratio = int(np.float32(g.rate) / np.float32(g.dt) + np.float32(0.5))
    nt_neg = int(round(abs(g.ot) / g.dt))
    rows = (g.nt - nt_neg - 1) // ratio + 1
    out = np.zeros(rows * nr, dtype=np.float32)
    fn = getattr(V.lib(), name)
    ctx.check(fn(ctx.handle, C.byref(g), V._p(V._f32(s.c11)), V._p(V._f32(s.c13)),
                 V._p(V._f32(s.c33)), V._p(V._f32(s.wavelet)), V._p(sloc), sloc.size // 4,
                 V._p(rloc), nr, V._p(V._f32(s.taper)), V._p(out)))
    return out


def _surveys():
    yield "g2_a", K.case2d("g2_a")["s"]
    # every step recorded (ratio 1, row 1 taken right after the source), 3 shots
    yield "ratio1", S.survey2d(nx=56, nz=36, nt=160, npad=8, d=10.0, dt=1e-3, rate=1e-3,
                               freq=20.0, src_x=250.0, src_z=40.0, rec_z=20.0, ns=3)


@pytest.mark.parametrize("which", ["g2_a", "ratio1"])
def test_noalloc_matches_synthetic_on_consecutive_calls(ctx, which):
    s = dict(_surveys())[which]
    g = s.geom()
    ref = _traces(ctx, "vti2d_synthetic", g, s)
    assert np.abs(ref).max() > 0
    first = _traces(ctx, "vti2d_synthetic_noalloc", g, s)
    second = _traces(ctx, "vti2d_synthetic_noalloc", g, s)
    assert rel_l2(first, ref) < TRACE_TOL
    assert rel_l2(second, ref) < TRACE_TOL


def test_noalloc_rejects_calls_beyond_its_array(ctx):
    # 1300 x 1300 padded grid: 8 * 1.69 M floats > the 10 Mi-float array
    nx = nz = 1280
    npad = 10
    n = (nx + 2 * npad) * (nz + 2 * npad)
    c = np.full(n, 4.0e6, dtype=np.float32)
    taper = np.ones(n, dtype=np.float32)
    wavelet = np.zeros(100, dtype=np.float32)
    sloc = np.array([100, 20, 1, 0], dtype=np.int32)
    rloc = np.array([200, 20], dtype=np.int32)
    g = V.Geom2d(nx=nx, nz=nz, nt=100, npad=npad, dx=10.0, dz=10.0, dt=1e-3, rate=2e-3, ot=0.0)
    out = np.zeros(50, dtype=np.float32)
    st = V.lib().vti2d_synthetic_noalloc(ctx.handle, C.byref(g), V._p(c), V._p(c), V._p(c),
                                         V._p(wavelet), V._p(sloc), 1, V._p(rloc), 1,
                                         V._p(taper), V._p(out))
    assert st == V.VTI_ERR_ARG
    assert b"static scratch" in V.lib().vti_ctx_last_error(ctx.handle)
    # the context stays usable
    s = K.case2d("g2_a")["s"]
    assert np.abs(_traces(ctx, "vti2d_synthetic_noalloc", s.geom(), s)).max() > 0


def _big_case(nx=980, nz=980, npad=10, nt=40, nrec=10):
    """A padded 1000 x 1000 grid: its 8 volumes (32 MB) are larger than any
    2D scratch the other tests grow, and still fit the static array."""
    n = (nx + 2 * npad) * (nz + 2 * npad)
    c33 = np.full(n, 4.0e6, dtype=np.float32)
    c11 = np.float32(1.2) * c33
    c13 = np.float32(1.05) * c33
    taper = np.ones(n, dtype=np.float32)
    wavelet = np.zeros(nt, dtype=np.float32)
    wavelet[:8] = np.hanning(8)
    sloc = np.array([500, 20, nrec, 0], dtype=np.int32)
    rloc = np.stack([np.arange(400, 400 + 10 * nrec, 10), np.full(nrec, 20)], 1)
    rloc = rloc.astype(np.int32).reshape(-1)
    g = V.Geom2d(nx=nx, nz=nz, nt=nt, npad=npad, dx=10.0, dz=10.0, dt=1e-3, rate=2e-3, ot=0.0)
    return g, (c11, c13, c33, wavelet, sloc, rloc, taper), nrec


def _call(ctx, g, arrays, nrec, rows):
    c11, c13, c33, wavelet, sloc, rloc, taper = arrays
    out = np.zeros(rows * nrec, dtype=np.float32)
    st = V.lib().vti2d_synthetic_noalloc(ctx.handle, C.byref(g), V._p(c11), V._p(c13),
                                         V._p(c33), V._p(wavelet), V._p(sloc), 1, V._p(rloc),
                                         nrec, V._p(taper), V._p(out))
    return st, out


def test_noalloc_allocates_no_device_memory(ctx):
    """The point of the entry point: after the first call on the device (which
    loads the kernels and looks up the array's address), a call on a grid
    larger than any earlier one leaves the device's free memory unchanged."""
    cudart = C.CDLL("libcudart.so.12")
    free, total = C.c_size_t(0), C.c_size_t(0)

    def free_bytes():
        assert cudart.cudaMemGetInfo(C.byref(free), C.byref(total)) == 0
        return free.value

    g, arrays, nrec = _big_case()
    rows = (g.nt - 1) // 2 + 1
    st, warm = _call(ctx, g, arrays, nrec, rows)
    assert st == V.VTI_OK
    before = free_bytes()
    st, again = _call(ctx, g, arrays, nrec, rows)
    after = free_bytes()
    assert st == V.VTI_OK
    np.testing.assert_array_equal(again, warm)
    # an allocating path would take >= 32 MB here
    assert abs(before - after) < (1 << 21), (before, after)


def test_noalloc_rejects_a_record_before_time_zero(ctx):
    """|ot| beyond the whole record leaves no trace rows: rejected before any
    work is queued, and the context stays usable."""
    s = K.case2d("g2_a")["s"]
    g = s.geom()
    g.ot = -float(g.nt + 50) * g.dt
    sloc = V._i32(s.sloc).reshape(-1)
    rloc = V._i32(s.rloc).reshape(-1)
    out = np.zeros(4, dtype=np.float32)
    for name in ("vti2d_synthetic_noalloc", "vti2d_synthetic"):
        st = getattr(V.lib(), name)(ctx.handle, C.byref(g), V._p(V._f32(s.c11)),
                                    V._p(V._f32(s.c13)), V._p(V._f32(s.c33)),
                                    V._p(V._f32(s.wavelet)), V._p(sloc), sloc.size // 4,
                                    V._p(rloc), rloc.size // 2, V._p(V._f32(s.taper)),
                                    V._p(out))
        assert st == V.VTI_ERR_ARG, name
        assert b"before time zero" in V.lib().vti_ctx_last_error(ctx.handle)
    g2 = s.geom()
    assert np.abs(_traces(ctx, "vti2d_synthetic_noalloc", g2, s)).max() > 0

