"""Python binding of libvti_b200.so (the C ABI declared in include/vti_b200.h).

The library is loaded from this directory. There is no fallback: if the
shared object is missing or fails to load, importing a compute entry point
raises. Arrays are numpy float32/int32 (host) or raw device pointers
(integers) tagged with ``MEM_DEVICE``.
"""
from __future__ import annotations

import atexit
import ctypes as C
import weakref
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libvti_b200.so"

VTI_OK = 0
VTI_ERR_ARG = 1
VTI_ERR_CFL = 2
VTI_ERR_OOM = 3
VTI_ERR_DEVICE = 4
VTI_ERR_TIMEOUT = 5
VTI_ERR_NONFINITE = 6
VTI_ERR_UNSUPPORTED = 7
VTI_ERR_BUSY = 8
JOB_MODEL = 0
JOB_GRADIENT = 1

MEM_HOST = 0
MEM_DEVICE = 1
OPT_FULL_STEPS = 1
OPT_CHECK_FINITE = 2
# observed-trace formats of Plan3d / Batch3d (set_trace_format)
TRACES_F32 = 0
TRACES_F16 = 1
# schedules of Batch3d.gradient
BATCH_AUTO = 0
BATCH_SIDE_BY_SIDE = 1
BATCH_PER_SHOT = 2


class VtiError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"vti status {status}: {msg}")
        self.status = status


class Geom3d(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("nt", C.c_int),
                ("npad", C.c_int), ("ox", C.c_float), ("oy", C.c_float), ("oz", C.c_float),
                ("ot", C.c_float), ("dx", C.c_float), ("dy", C.c_float), ("dz", C.c_float),
                ("dt", C.c_float), ("sampling_rate", C.c_float)]


class Job3d(C.Structure):
    """vti3d_job: one request of the 3D serving engine."""
    _fields_ = [("kind", C.c_int), ("g", Geom3d), ("c11", C.c_void_p), ("c13", C.c_void_p),
                ("c33", C.c_void_p), ("wavelet", C.c_void_p), ("souloc", C.c_void_p),
                ("recloc", C.c_void_p), ("nrec", C.c_int), ("dobs", C.c_void_p),
                ("randb", C.c_void_p), ("seed", C.c_uint)]


class Geom2d(C.Structure):
    _fields_ = [("nx", C.c_int), ("nz", C.c_int), ("nt", C.c_int), ("npad", C.c_int),
                ("dx", C.c_float), ("dz", C.c_float), ("dt", C.c_float), ("rate", C.c_float),
                ("ot", C.c_float)]


_lib = None

F32P = C.POINTER(C.c_float)
I32P = C.POINTER(C.c_int)
VP = C.c_void_p


def _signatures():
    P = VP
    return {
        "vti_ctx_create": (C.c_int, [C.c_int, C.POINTER(VP)]),
        "vti_ctx_destroy": (C.c_int, [P]),
        "vti_status_string": (C.c_char_p, [C.c_int]),
        "vti_ctx_last_error": (C.c_char_p, [P]),
        "vti_ctx_stream": (VP, [P]),
        "vti_ctx_kernel_launches": (C.c_uint64, [P]),
        "vti_ctx_set_timing": (C.c_int, [P, C.c_int]),
        "vti_ctx_set_plan_cache": (C.c_int, [P, C.c_int]),
        "vti_ctx_set_2d_resident": (C.c_int, [P, C.c_int]),
        "vti_ctx_kernel_time": (C.c_int, [P, C.c_char_p, C.POINTER(C.c_double),
                                          C.POINTER(C.c_uint64)]),
        "vti3d_cfl_number": (C.c_double, [P, P, P, P]),
        "vti2d_cfl_number": (C.c_double, [P, P, P, P]),
        "vti_ctx_check_bounded_wait": (C.c_int, [P, C.c_uint]),
        "vti3d_get_boundary": (None, [P, P, C.c_int, C.c_int, C.c_int, C.c_int]),
        "vti3d_put_boundary": (None, [P, P, C.c_int, C.c_int, C.c_int, C.c_int]),
        "vti3d_zero_boundary": (None, [P, C.c_int, C.c_int, C.c_int, C.c_int]),
        "vti_vepsdel_to_cij": (None, [P] * 6 + [C.c_float] * 3 + [C.c_size_t]),
        "vti_grad_cij_to_vepsdel": (None, [P] * 9 + [C.c_float] * 3 + [C.c_size_t]),
        "vti_dvepsdel_to_dcij": (None, [P] * 12 + [C.c_float] * 3 + [C.c_size_t]),
        "vti_check_eps_del": (C.c_int, [P, P, C.c_float, C.c_float, C.c_size_t, P]),
        "vti3d_plan_create": (C.c_int, [P, P, C.c_uint, C.POINTER(VP)]),
        "vti3d_plan_destroy": (C.c_int, [P]),
        "vti3d_plan_set_model": (C.c_int, [P, P, P, P, P, P, C.c_int]),
        "vti3d_plan_set_wavelet": (C.c_int, [P, P, C.c_int]),
        "vti3d_plan_set_receivers": (C.c_int, [P, P, C.c_int]),
        "vti3d_plan_model_data": (C.c_int, [P, P, P, C.c_int, P, C.c_int]),
        "vti3d_plan_gradient": (C.c_int, [P, P, P, C.c_int, P, C.c_int, P, C.c_int,
                                          C.POINTER(C.c_double)]),
        "vti3d_plan_objfunc": (C.c_int, [P, P, P, C.c_int, P, C.c_int, C.POINTER(C.c_double)]),
        "vti3d_plan_rtm": (C.c_int, [P, P, P, C.c_int, P, C.c_int, P, C.c_int]),
        "vti3d_plan_odcig": (C.c_int, [P, P, P, C.c_int, P, C.c_int, C.c_int, P, C.c_int]),
        "vti3d_plan_set_misfit": (C.c_int, [P, C.c_float, C.c_int, C.c_int]),
        "vti3d_rtm_cij": (C.c_int, [P, P, P, P, P, P, P, P, C.c_int, P, C.c_int, P, P, C.c_uint]),
        "vti3d_plan_wavefield": (VP, [P]),
        "vti3d_model_data_cij": (C.c_int, [P, P, P, P, P, P, P, P, C.c_int, P, C.c_int, P,
                                           C.c_uint]),
        "vti3d_gradient_cij": (C.c_int, [P, P, P, P, P, P, P, P, C.c_int, P, C.c_int, P, P,
                                         C.POINTER(C.c_double), C.c_uint]),
        "vti2d_synthetic": (C.c_int, [P, P, P, P, P, P, P, C.c_int, P, C.c_int, P, P]),
        "vti2d_synthetic_noalloc": (C.c_int, [P, P, P, P, P, P, P, C.c_int, P, C.c_int, P, P]),
        "vti2d_modeling": (C.c_int, [P, P, P, P, P, P, C.c_int, P, P]),
        "vti2d_init_taper": (None, [P, C.c_int, C.c_int, C.c_int]),
        "vti_random_boundary": (C.c_int, [P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float,
                                          C.c_int, C.c_float, C.c_float]),
        "vti2d_gradient": (C.c_int, [P] * 11 + [C.c_int, P, C.c_int, P, C.POINTER(C.c_double)]),
        "vti2d_gn_hessian": (C.c_int, [P] * 13 + [C.c_int, P, C.c_int, P]),
        "vti2d_rtm": (C.c_int, [P] * 9 + [C.c_int, P, C.c_int, P]),
        "vti2d_wavelet_gradient": (C.c_int, [P] * 8 + [C.c_int, P, C.c_int, P]),
        "vti2d_odcig": (C.c_int, [P, P, C.c_int] + [P] * 7 + [C.c_int, P, C.c_int, P]),
        "vti3d_plan_wavelet_gradient": (C.c_int, [P, P, P, C.c_int, P, C.c_int, P, C.c_int]),
        "vti3d_wavelet_gradient_cij": (C.c_int, [P] * 7 + [C.c_int, P, C.c_int, P, P, C.c_uint]),
        "vti3d_plan_get_wavefield": (C.c_int, [P, P, C.c_int]),
        "vti3d_gradient_vepsdel": (C.c_int, [P, P, P, P, P, P, P, C.c_float, C.c_float,
                                             C.c_float, P, P, P, C.c_int, P, C.c_int, P, P, P, P,
                                             C.POINTER(C.c_double), C.c_uint]),
        "vti3d_batch_create": (C.c_int, [P, P, C.c_uint, C.POINTER(VP)]),
        "vti3d_batch_destroy": (C.c_int, [P]),
        "vti3d_batch_set_model": (C.c_int, [P, P, P, P, C.c_int]),
        "vti3d_batch_set_wavelet": (C.c_int, [P, P, C.c_int]),
        "vti3d_batch_set_receivers": (C.c_int, [P, P, C.c_int]),
        "vti3d_batch_set_shots": (C.c_int, [P, C.c_int, P, P, C.c_uint]),
        "vti3d_batch_set_options": (C.c_int, [P, C.c_int, C.c_int, C.c_int]),
        "vti3d_batch_autotune": (C.c_int, [P, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "vti3d_batch_set_schedule": (C.c_int, [P, C.c_int]),
        "vti3d_batch_set_trace_format": (C.c_int, [P, C.c_int]),
        "vti3d_plan_set_trace_format": (C.c_int, [P, C.c_int]),
        "vti_traces_f16_bytes": (C.c_size_t, [C.c_int, C.c_int]),
        "vti_traces_pack_f16": (C.c_int, [P, C.c_int, C.c_int, P]),
        "vti_traces_unpack_f16": (C.c_int, [P, C.c_int, C.c_int, P]),
        "vti3d_batch_get_schedule": (C.c_int, [P, C.POINTER(C.c_int)]),
        "vti3d_batch_gradient": (C.c_int, [P, P, C.c_int, P, C.c_int, C.POINTER(C.c_double)]),
        "vti3d_batch_get_shot_models": (C.c_int, [P, C.c_int, P, P]),
        "vti3d_gnhv_exact": (C.c_int, [P] * 9 + [C.c_int, P, C.c_int, C.c_uint, P, P,
                                               C.POINTER(C.c_double), P, P]),
        "vti3d_engine_job_bytes": (C.c_size_t, [P]),
        "vti3d_engine_create": (C.c_int, [P, C.c_size_t, C.POINTER(VP)]),
        "vti3d_engine_destroy": (C.c_int, [P]),
        "vti3d_engine_submit": (C.c_int, [P, P, C.POINTER(C.c_int)]),
        "vti3d_engine_step": (C.c_int, [P, C.c_int, C.POINTER(C.c_int)]),
        "vti3d_engine_poll": (C.c_int, [P, P, C.c_int, C.POINTER(C.c_int)]),
        "vti3d_engine_result": (C.c_int, [P, C.c_int, P, C.POINTER(C.c_double)]),
        "vti3d_engine_cancel": (C.c_int, [P, C.c_int]),
        "vti3d_engine_stats": (C.c_int, [P, C.POINTER(C.c_size_t), C.POINTER(C.c_int),
                                         C.POINTER(C.c_int)]),
    }


def _declare(lib):
    for name, (res, args) in _signatures().items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args


def exported_symbols():
    """Names of every C-ABI entry point this binding declares."""
    return sorted(_signatures())


def lib():
    """Load (once) and return the shared library; raises if it is missing."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: run `make -C thesis-source-code_b200` "
                              "(or __graft_entry__.build())")
        lib_ = C.CDLL(str(LIB_PATH))
        _declare(lib_)
        _lib = lib_
    return _lib


def _p(a):
    """ctypes pointer of a contiguous numpy array, a raw int pointer, or None."""
    if a is None:
        return None
    if isinstance(a, int):
        return C.c_void_p(a)
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("array must be C-contiguous")
    # data_as keeps a reference to the array: a converted temporary such as
    # _f32(x) stays alive until the foreign call that receives it returns
    return a.ctypes.data_as(C.c_void_p)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _obs(a):
    """Observed traces for a plan or batch call: FP32 traces, or a packed
    16-bit block (uint8 array from pack_traces_f16) passed through as is."""
    if isinstance(a, np.ndarray) and a.dtype == np.uint8:
        return np.ascontiguousarray(a)
    return _f32(a)


def traces_f16_bytes(nr: int, nnt: int) -> int:
    return int(lib().vti_traces_f16_bytes(nr, nnt))


def pack_traces_f16(traces, nnt: int):
    """FP32 traces (nr x nnt, trace-major) -> a VTI_TRACES_F16 block (uint8):
    nnt FP32 plane scales, then the traces as IEEE halves."""
    t = _f32(traces).reshape(-1)
    nr = t.size // nnt
    block = np.zeros(traces_f16_bytes(nr, nnt), dtype=np.uint8)
    st = lib().vti_traces_pack_f16(_p(t), nr, nnt, _p(block))
    if st != VTI_OK:
        raise VtiError(st, "vti_traces_pack_f16 failed")
    return block


def unpack_traces_f16(block, nr: int, nnt: int):
    """The FP32 traces (nr * nnt) a VTI_TRACES_F16 block stands for."""
    out = np.zeros(nr * nnt, dtype=np.float32)
    st = lib().vti_traces_unpack_f16(_p(np.ascontiguousarray(block)), nr, nnt, _p(out))
    if st != VTI_OK:
        raise VtiError(st, "vti_traces_unpack_f16 failed")
    return out


_contexts = weakref.WeakSet()


@atexit.register
def _close_contexts():
    """Closes every live context (its plans, batches and engines first) while
    the interpreter and the CUDA runtime are still whole; left to garbage
    collection at shutdown, a handle could be destroyed after the library
    that owns it."""
    for c in list(_contexts):
        try:
            c.close()
        except Exception:
            pass


class Context:
    """One CUDA device. Mirrors vti_ctx_create/destroy."""

    def __init__(self, device: int = 0):
        self._h = VP()
        self._plans = weakref.WeakSet()  # plans must be destroyed before the context
        st = lib().vti_ctx_create(device, C.byref(self._h))
        if st != VTI_OK:
            raise VtiError(st, "vti_ctx_create failed (no CUDA device?)")
        _contexts.add(self)

    @property
    def handle(self):
        return self._h

    def check(self, st: int):
        if st != VTI_OK:
            msg = lib().vti_ctx_last_error(self._h) or lib().vti_status_string(st)
            raise VtiError(st, msg.decode() if isinstance(msg, bytes) else str(msg))

    @property
    def stream(self) -> int:
        return lib().vti_ctx_stream(self._h) or 0

    @property
    def launches(self) -> int:
        return int(lib().vti_ctx_kernel_launches(self._h))

    def set_timing(self, enable: bool):
        self.check(lib().vti_ctx_set_timing(self._h, 1 if enable else 0))

    def set_2d_resident(self, enable: bool):
        """Shared-memory resident 2D traces where the grid fits one cluster (default)."""
        self.check(lib().vti_ctx_set_2d_resident(self._h, 1 if enable else 0))

    def set_plan_cache(self, enable: bool):
        """Keep (default) or free the plan of the one-call 3D forms between calls."""
        self.check(lib().vti_ctx_set_plan_cache(self._h, 1 if enable else 0))

    def kernel_time(self, kernel: str):
        """(total device ms, launches) of a timed kernel: fwd3d, bwd3d, step2d."""
        ms, cnt = C.c_double(0), C.c_uint64(0)
        self.check(lib().vti_ctx_kernel_time(self._h, kernel.encode(), C.byref(ms),
                                             C.byref(cnt)))
        return ms.value, int(cnt.value)

    def synchronize(self):
        self.kernel_time("fwd3d")

    def close(self):
        if self._h:
            for p in list(self._plans):
                p.close()
            lib().vti_ctx_destroy(self._h)
            self._h = VP()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def geom3d(nx, ny, nz, nt, npad, dx, dy, dz, dt, sampling_rate, ox=0.0, oy=0.0, oz=0.0, ot=0.0):
    return Geom3d(nx, ny, nz, nt, npad, ox, oy, oz, ot, dx, dy, dz, dt, sampling_rate)


def geom2d(nx, nz, nt, npad, dx, dz, dt, rate, ot=0.0):
    return Geom2d(nx, nz, nt, npad, dx, dz, dt, rate, ot)


def nnt3d(g: Geom3d) -> int:
    s = int(np.round(np.float32(g.sampling_rate) / np.float32(g.dt)))
    return (g.nt - 1) // s + 1


class Plan3d:
    """Device-resident 3D plan (vti3d_plan_*)."""

    def __init__(self, ctx: Context, g: Geom3d, flags: int = 0):
        self.ctx, self.g = ctx, g
        self._h = VP()
        ctx.check(lib().vti3d_plan_create(ctx.handle, C.byref(g), flags, C.byref(self._h)))
        ctx._plans.add(self)

    def set_model(self, c11, c13, c33, padb=None, randb=None, mem=MEM_HOST):
        if mem == MEM_HOST:
            c11, c13, c33 = _f32(c11), _f32(c13), _f32(c33)
            padb = None if padb is None else _f32(padb)
            randb = None if randb is None else _f32(randb)
            self._keep = (c11, c13, c33, padb, randb)
        self.ctx.check(lib().vti3d_plan_set_model(self._h, _p(c11), _p(c13), _p(c33), _p(padb),
                                                  _p(randb), mem))

    def set_wavelet(self, w, mem=MEM_HOST):
        if mem == MEM_HOST:
            w = _f32(w)
        self.ctx.check(lib().vti3d_plan_set_wavelet(self._h, _p(w), mem))

    def set_receivers(self, recloc):
        recloc = _f32(recloc).reshape(-1)
        self.ctx.check(lib().vti3d_plan_set_receivers(self._h, _p(recloc), recloc.size // 4))

    def model_data(self, souloc, shotid, out=None, mem=MEM_HOST, nrec_total=None):
        souloc, shotid = _f32(souloc).reshape(-1), _i32(shotid)
        if out is None:
            nr = nrec_total if nrec_total is not None else int(
                max(souloc[5 * s + 3] + souloc[5 * s + 4] for s in shotid))
            out = np.zeros(nnt3d(self.g) * nr, dtype=np.float32)
        self.ctx.check(lib().vti3d_plan_model_data(self._h, _p(souloc), _p(shotid), len(shotid),
                                                   _p(out), mem))
        return out

    def gradient(self, souloc, shotid, dobs, dobs_mem=MEM_HOST, fgcij=None, fgcij_mem=MEM_HOST):
        souloc, shotid = _f32(souloc).reshape(-1), _i32(shotid)
        if dobs_mem == MEM_HOST:
            dobs = _obs(dobs)
        n = self.g.nx * self.g.ny * self.g.nz
        if fgcij is None:
            fgcij = np.zeros(1 + 3 * n, dtype=np.float32)
        mis = C.c_double(0)
        self.ctx.check(lib().vti3d_plan_gradient(self._h, _p(souloc), _p(shotid), len(shotid),
                                                 _p(dobs), dobs_mem, _p(fgcij), fgcij_mem,
                                                 C.byref(mis)))
        return fgcij, mis.value

    def set_trace_format(self, fmt):
        """TRACES_F32 (default) or TRACES_F16: observed data passed as a block
        from pack_traces_f16 (host or device memory)."""
        self.ctx.check(lib().vti3d_plan_set_trace_format(self._h, int(fmt)))

    def set_misfit(self, tpow=0.0, objtype=0, halfwidth=20):
        """tpow gain / AGC misfit of the gradient (the reference's tpow=,
        objtype=, halfwidth= parameters)."""
        self.ctx.check(lib().vti3d_plan_set_misfit(self._h, tpow, objtype, halfwidth))

    def rtm(self, souloc, shotid, data, data_mem=MEM_HOST, image=None, image_mem=MEM_HOST):
        """rtmCij3d_f on the resident model: the image (nxyz)."""
        souloc, shotid = _f32(souloc).reshape(-1), _i32(shotid)
        if data_mem == MEM_HOST:
            data = _obs(data)
        if image is None:
            image = np.zeros(self.g.nx * self.g.ny * self.g.nz, dtype=np.float32)
        self.ctx.check(lib().vti3d_plan_rtm(self._h, _p(souloc), _p(shotid), len(shotid),
                                            _p(data), data_mem, _p(image), image_mem))
        return image

    def odcig(self, souloc, shotid, data, nlag, data_mem=MEM_HOST):
        """odcig3d_f on the resident model: (2 nlag + 1, nxyz) gathers, lag -nlag first."""
        souloc, shotid = _f32(souloc).reshape(-1), _i32(shotid)
        if data_mem == MEM_HOST:
            data = _obs(data)
        n = self.g.nx * self.g.ny * self.g.nz
        image = np.zeros((2 * nlag + 1) * n, dtype=np.float32)
        self.ctx.check(lib().vti3d_plan_odcig(self._h, _p(souloc), _p(shotid), len(shotid),
                                              _p(data), data_mem, int(nlag), _p(image),
                                              MEM_HOST))
        return image.reshape(2 * nlag + 1, n)

    def objfunc(self, souloc, shotid, dobs, dobs_mem=MEM_HOST):
        souloc, shotid = _f32(souloc).reshape(-1), _i32(shotid)
        if dobs_mem == MEM_HOST:
            dobs = _obs(dobs)
        mis = C.c_double(0)
        self.ctx.check(lib().vti3d_plan_objfunc(self._h, _p(souloc), _p(shotid), len(shotid),
                                                _p(dobs), dobs_mem, C.byref(mis)))
        return mis.value

    def wavefield_ptr(self) -> int:
        return lib().vti3d_plan_wavefield(self._h) or 0

    def close(self):
        if self._h:
            lib().vti3d_plan_destroy(self._h)
            self._h = VP()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch3d:
    """Batched multi-shot 3D gradient (vti3d_batch_*): every shot on its own
    window of the model, all shots advanced by one forward and one backward
    launch per time step."""

    def __init__(self, ctx: Context, g: Geom3d, flags: int = 0):
        self.ctx, self.g = ctx, g
        self._h = VP()
        ctx.check(lib().vti3d_batch_create(ctx.handle, C.byref(g), flags, C.byref(self._h)))
        ctx._plans.add(self)
        self.windows = []

    def set_model(self, c11, c13, c33, mem=MEM_HOST):
        if mem == MEM_HOST:
            c11, c13, c33 = _f32(c11), _f32(c13), _f32(c33)
        self.ctx.check(lib().vti3d_batch_set_model(self._h, _p(c11), _p(c13), _p(c33), mem))

    def set_wavelet(self, w, mem=MEM_HOST):
        if mem == MEM_HOST:
            w = _f32(w)
        self.ctx.check(lib().vti3d_batch_set_wavelet(self._h, _p(w), mem))

    def set_receivers(self, recloc):
        recloc = _f32(recloc).reshape(-1)
        self.ctx.check(lib().vti3d_batch_set_receivers(self._h, _p(recloc), recloc.size // 4))

    def set_shots(self, souloc, windows, seed=0):
        """souloc: 5 floats per shot; windows: (x0, y0, nx, ny) per shot."""
        souloc = _f32(souloc).reshape(-1)
        w = np.ascontiguousarray(np.asarray(windows, dtype=np.int32).reshape(-1, 4))
        self.windows = [tuple(int(v) for v in r) for r in w]
        self.ctx.check(lib().vti3d_batch_set_shots(self._h, len(w), _p(souloc), _p(w),
                                                   seed & 0xffffffff))

    def set_options(self, use_graph=False, seg_fwd=0, seg_bwd=0):
        self.ctx.check(lib().vti3d_batch_set_options(self._h, int(use_graph), seg_fwd, seg_bwd))

    def autotune(self):
        a, b = C.c_int(0), C.c_int(0)
        self.ctx.check(lib().vti3d_batch_autotune(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def set_trace_format(self, fmt):
        """TRACES_F32 (default) or TRACES_F16 (a pack_traces_f16 block over all
        receivers)."""
        self.ctx.check(lib().vti3d_batch_set_trace_format(self._h, int(fmt)))

    def set_schedule(self, schedule):
        """BATCH_AUTO, BATCH_SIDE_BY_SIDE or BATCH_PER_SHOT."""
        self.ctx.check(lib().vti3d_batch_set_schedule(self._h, int(schedule)))

    @property
    def schedule(self):
        """The schedule the next gradient runs (auto resolved)."""
        v = C.c_int(0)
        self.ctx.check(lib().vti3d_batch_get_schedule(self._h, C.byref(v)))
        return v.value

    def gradient(self, dobs, dobs_mem=MEM_HOST, fgcij=None, fgcij_mem=MEM_HOST):
        if dobs_mem == MEM_HOST:
            dobs = _obs(dobs)
        n = self.g.nx * self.g.ny * self.g.nz
        if fgcij is None:
            fgcij = np.zeros(1 + 3 * n, dtype=np.float32)
        mis = C.c_double(0)
        self.ctx.check(lib().vti3d_batch_gradient(self._h, _p(dobs), dobs_mem, _p(fgcij),
                                                  fgcij_mem, C.byref(mis)))
        return fgcij, mis.value

    def shot_models(self, k):
        """(pad-boundary, random-boundary) window models of shot k, 3*n each."""
        x0, y0, nx, ny = self.windows[k]
        n = nx * ny * self.g.nz
        cpad = np.zeros(3 * n, dtype=np.float32)
        crand = np.zeros(3 * n, dtype=np.float32)
        self.ctx.check(lib().vti3d_batch_get_shot_models(self._h, k, _p(cpad), _p(crand)))
        return cpad, crand

    def close(self):
        if self._h:
            lib().vti3d_batch_destroy(self._h)
            self._h = VP()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Engine3d:
    """3D serving engine (vti3d_engine_*): continuous batching of modeling and
    gradient jobs of different grids under a device byte budget."""

    def __init__(self, ctx: Context, max_bytes: int):
        self.ctx = ctx
        self._h = VP()
        ctx.check(lib().vti3d_engine_create(ctx.handle, int(max_bytes), C.byref(self._h)))
        ctx._plans.add(self)
        self._jobs = {}

    @staticmethod
    def make_job(kind, g, c11, c13, c33, wavelet, souloc, recloc, dobs=None, randb=None,
                 seed=0):
        keep = [_f32(a) for a in (c11, c13, c33, wavelet, souloc, recloc)]
        keep.append(None if dobs is None else _f32(dobs))
        keep.append(None if randb is None else _f32(randb))
        j = Job3d(kind, g, *[None if a is None else a.ctypes.data for a in keep[:6]],
                  keep[5].size // 4, None if keep[6] is None else keep[6].ctypes.data,
                  None if keep[7] is None else keep[7].ctypes.data, seed & 0xffffffff)
        j._keep = keep
        return j

    def job_bytes(self, job):
        return int(lib().vti3d_engine_job_bytes(C.byref(job)))

    def submit(self, job):
        """Job id, or None when the memory budget is full (VTI_ERR_BUSY)."""
        jid = C.c_int(0)
        st = lib().vti3d_engine_submit(self._h, C.byref(job), C.byref(jid))
        if st == VTI_ERR_BUSY:
            return None
        self.ctx.check(st)
        self._jobs[jid.value] = job
        return jid.value

    def step(self, ticks):
        n = C.c_int(0)
        self.ctx.check(lib().vti3d_engine_step(self._h, int(ticks), C.byref(n)))
        return n.value

    def poll(self, max_ids=256):
        ids = np.zeros(max_ids, dtype=np.int32)
        n = C.c_int(0)
        self.ctx.check(lib().vti3d_engine_poll(self._h, _p(ids), max_ids, C.byref(n)))
        return [int(i) for i in ids[:n.value]]

    def result(self, jid):
        job = self._jobs.pop(jid)
        g = job.g
        if job.kind == JOB_MODEL:
            out = np.zeros(nnt3d(g) * job.nrec, dtype=np.float32)
        else:
            out = np.zeros(1 + 3 * g.nx * g.ny * g.nz, dtype=np.float32)
        mis = C.c_double(0)
        self.ctx.check(lib().vti3d_engine_result(self._h, jid, _p(out), C.byref(mis)))
        return out, mis.value

    def cancel(self, jid):
        """Drops an admitted job (vti3d_engine_cancel)."""
        self.ctx.check(lib().vti3d_engine_cancel(self._h, int(jid)))
        self._jobs.pop(jid, None)

    def stats(self):
        u, n, t = C.c_size_t(0), C.c_int(0), C.c_int(0)
        self.ctx.check(lib().vti3d_engine_stats(self._h, C.byref(u), C.byref(n), C.byref(t)))
        return u.value, n.value, t.value

    def close(self):
        if self._h:
            lib().vti3d_engine_destroy(self._h)
            self._h = VP()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


GNHV_BF16 = 1
GNHV_BF16_SR = 2  # with GNHV_BF16: stochastic rounding (default: nearest)


def gnhv_exact(ctx, g: Geom3d, c11, c13, c33, wavelet, souloc, recloc, dc=None, dobs=None,
               checkpoint_every=0, want=("hv", "grad", "traces", "born"), flags=0):
    """vti3d_gnhv_exact: exact-mode Gauss-Newton product H dc, gradient,
    misfit and traces of one shot. Returns a dict of the requested outputs."""
    n = g.nx * g.ny * g.nz
    recloc = _f32(recloc).reshape(-1)
    nrec = recloc.size // 4
    nnt = nnt3d(g)
    out = {}
    hv = np.zeros(3 * n, dtype=np.float32) if "hv" in want and dc is not None else None
    grad = np.zeros(3 * n, dtype=np.float32) if "grad" in want and dobs is not None else None
    tr = np.zeros(nnt * nrec, dtype=np.float32) if "traces" in want else None
    born = np.zeros(nnt * nrec, dtype=np.float32) if "born" in want and dc is not None else None
    mis = C.c_double(0)
    args = [_f32(c11), _f32(c13), _f32(c33), None if dc is None else _f32(dc), _f32(wavelet),
            _f32(souloc), recloc]
    dobs_ = None if dobs is None else _f32(dobs)
    ctx.check(lib().vti3d_gnhv_exact(ctx.handle, C.byref(g), *[_p(a) for a in args], nrec,
                                     _p(dobs_), checkpoint_every, flags, _p(hv), _p(grad),
                                     C.byref(mis) if dobs is not None else None, _p(tr),
                                     _p(born)))
    for k, v in (("hv", hv), ("grad", grad), ("traces", tr), ("born", born)):
        if v is not None:
            out[k] = v
    if dobs is not None:
        out["misfit"] = mis.value
    return out


# ------------------------------------------------------- reference-named API
def modelDataCij3d_f(ctx, g: Geom3d, souloc, shotid, recloc, wavelet, c11, c13, c33, flags=0):
    """modelDataCij3d_f (lib/vti-fwi-3d/gpu/modelData3d_f.cu:427): returns ddata."""
    souloc, recloc = _f32(souloc).reshape(-1), _f32(recloc).reshape(-1)
    shotid = _i32(shotid)
    nrtot = recloc.size // 4
    out = np.zeros(nnt3d(g) * nrtot, dtype=np.float32)
    ctx.check(lib().vti3d_model_data_cij(ctx.handle, C.byref(g), _p(_f32(c11)), _p(_f32(c13)),
                                         _p(_f32(c33)), _p(_f32(wavelet)), _p(souloc),
                                         _p(shotid), len(shotid), _p(recloc), nrtot, _p(out),
                                         flags))
    return out


def rtmCij3d_f(ctx, g: Geom3d, souloc, shotid, recloc, wavelet, c11, c13, c33, data, flags=0):
    """rtmCij3d_f (lib/vti-fwi-3d/gpu/rtm3d_f.cu:161): returns the image (nxyz)."""
    souloc, recloc = _f32(souloc).reshape(-1), _f32(recloc).reshape(-1)
    shotid = _i32(shotid)
    out = np.zeros(g.nx * g.ny * g.nz, dtype=np.float32)
    ctx.check(lib().vti3d_rtm_cij(ctx.handle, C.byref(g), _p(_f32(c11)), _p(_f32(c13)),
                                  _p(_f32(c33)), _p(_f32(wavelet)), _p(souloc), _p(shotid),
                                  len(shotid), _p(recloc), recloc.size // 4, _p(_f32(data)),
                                  _p(out), flags))
    return out


def objFuncGradientCij3d_f(ctx, g: Geom3d, souloc, shotid, recloc, wavelet, cij, padb, randb,
                           dobs, flags=0):
    """objFuncGradientCij3d_f (objFuncGradient3d_f.cu:361): returns (fgcij, misfit64)."""
    souloc, recloc = _f32(souloc).reshape(-1), _f32(recloc).reshape(-1)
    shotid = _i32(shotid)
    n = g.nx * g.ny * g.nz
    fg = np.zeros(1 + 3 * n, dtype=np.float32)
    mis = C.c_double(0)
    ctx.check(lib().vti3d_gradient_cij(
        ctx.handle, C.byref(g), _p(_f32(cij)), _p(None if padb is None else _f32(padb)),
        _p(None if randb is None else _f32(randb)), _p(_f32(wavelet)), _p(souloc), _p(shotid),
        len(shotid), _p(recloc), recloc.size // 4, _p(_f32(dobs)), _p(fg), C.byref(mis), flags))
    return fg, mis.value


def synthetic_f(ctx, g: Geom2d, c11, c13, c33, wavelet, sloc, rloc, taper):
    """synthetic_f (lib/vti-fwi-2d/synthetic_f.cu:13): data[(it/ratio)*nr + ir]."""
    sloc, rloc = _i32(sloc).reshape(-1), _i32(rloc).reshape(-1)
    nr = rloc.size // 2
    ratio = int(np.float32(g.rate) / np.float32(g.dt) + np.float32(0.5))
    nt_neg = int(round(abs(g.ot) / g.dt))
    rows = (g.nt - nt_neg - 1) // ratio + 1
    out = np.zeros(rows * nr, dtype=np.float32)
    ctx.check(lib().vti2d_synthetic(ctx.handle, C.byref(g), _p(_f32(c11)), _p(_f32(c13)),
                                    _p(_f32(c33)), _p(_f32(wavelet)), _p(sloc), sloc.size // 4,
                                    _p(rloc), nr, _p(_f32(taper)), _p(out)))
    return out.reshape(rows, nr)


def objFuncGradient_f(ctx, g: Geom2d, data, c11, c13, c33, wavelet, sloc, rloc, taper):
    """objFuncGradient_f (lib/vti-fwi-2d/objFuncGradient_f.cu:15): (gc11, gc13, gc33, f)."""
    sloc, rloc = _i32(sloc).reshape(-1), _i32(rloc).reshape(-1)
    n = (g.nx + 2 * g.npad) * (g.nz + 2 * g.npad)
    out = [np.zeros(n, dtype=np.float32) for _ in range(3)]
    mis = C.c_double(0)
    ctx.check(lib().vti2d_gradient(ctx.handle, C.byref(g), _p(out[0]), _p(out[1]), _p(out[2]),
                                   _p(_f32(data)), _p(_f32(c11)), _p(_f32(c13)), _p(_f32(c33)),
                                   _p(_f32(wavelet)), _p(sloc), sloc.size // 4, _p(rloc),
                                   rloc.size // 2, _p(_f32(taper)), C.byref(mis)))
    return out[0], out[1], out[2], mis.value


def odcig_f(ctx, g: Geom2d, nhx, data, c11, c13, c33, wavelet, sloc, rloc, taper):
    """odcig_f (lib/vti-fwi-2d/odcig_f.cu:12): (2 nhx + 1) x nnxz gathers."""
    sloc, rloc = _i32(sloc).reshape(-1), _i32(rloc).reshape(-1)
    nnxz = (g.nx + 2 * g.npad) * (g.nz + 2 * g.npad)
    out = np.zeros((2 * nhx + 1) * nnxz, dtype=np.float32)
    ctx.check(lib().vti2d_odcig(ctx.handle, C.byref(g), nhx, _p(out), _p(_f32(data)),
                                _p(_f32(c11)), _p(_f32(c13)), _p(_f32(c33)), _p(_f32(wavelet)),
                                _p(sloc), sloc.size // 4, _p(rloc), rloc.size // 2,
                                _p(_f32(taper))))
    return out.reshape(2 * nhx + 1, nnxz)


def waveletGradient_f(ctx, g: Geom2d, data, c11, c13, c33, sloc, rloc, taper):
    """waveletGradient_f (lib/vti-fwi-2d/objFuncGradient_f.cu:373): nt floats."""
    sloc, rloc = _i32(sloc).reshape(-1), _i32(rloc).reshape(-1)
    out = np.zeros(g.nt, dtype=np.float32)
    ctx.check(lib().vti2d_wavelet_gradient(ctx.handle, C.byref(g), _p(out), _p(_f32(data)),
                                           _p(_f32(c11)), _p(_f32(c13)), _p(_f32(c33)),
                                           _p(sloc), sloc.size // 4, _p(rloc), rloc.size // 2,
                                           _p(_f32(taper))))
    return out


def waveletGradientCij3d_f(ctx, g: Geom3d, souloc, shotid, recloc, c11, c13, c33, data,
                           flags=0):
    """waveletGradientCij3d_f (lib/vti-fwi-3d/gpu/modelData3d_f.cu:858): nt floats."""
    souloc, recloc = _f32(souloc).reshape(-1), _f32(recloc).reshape(-1)
    shotid = _i32(shotid)
    out = np.zeros(g.nt, dtype=np.float32)
    ctx.check(lib().vti3d_wavelet_gradient_cij(ctx.handle, C.byref(g), _p(_f32(c11)),
                                               _p(_f32(c13)), _p(_f32(c33)), _p(souloc),
                                               _p(shotid), len(shotid), _p(recloc),
                                               recloc.size // 4, _p(_f32(data)), _p(out), flags))
    return out


def rtm_f(ctx, g: Geom2d, data, c11, c13, c33, wavelet, sloc, rloc, taper):
    """rtm_f (lib/vti-fwi-2d/rtm_f.cu:13): the migrated image (nnxz)."""
    sloc, rloc = _i32(sloc).reshape(-1), _i32(rloc).reshape(-1)
    out = np.zeros((g.nx + 2 * g.npad) * (g.nz + 2 * g.npad), dtype=np.float32)
    ctx.check(lib().vti2d_rtm(ctx.handle, C.byref(g), _p(out), _p(_f32(data)), _p(_f32(c11)),
                              _p(_f32(c13)), _p(_f32(c33)), _p(_f32(wavelet)), _p(sloc),
                              sloc.size // 4, _p(rloc), rloc.size // 2, _p(_f32(taper))))
    return out


def GNhessian_f(ctx, g: Geom2d, c11, c13, c33, dc11, dc13, dc33, wavelet, sloc, rloc, taper):
    """GNhessian_f (lib/vti-fwi-2d/hessian_f.cu:575): Gauss-Newton H * dc."""
    sloc, rloc = _i32(sloc).reshape(-1), _i32(rloc).reshape(-1)
    n = (g.nx + 2 * g.npad) * (g.nz + 2 * g.npad)
    out = [np.zeros(n, dtype=np.float32) for _ in range(3)]
    ctx.check(lib().vti2d_gn_hessian(ctx.handle, C.byref(g), _p(out[0]), _p(out[1]),
                                     _p(out[2]), _p(_f32(c11)), _p(_f32(c13)), _p(_f32(c33)),
                                     _p(_f32(dc11)), _p(_f32(dc13)), _p(_f32(dc33)),
                                     _p(_f32(wavelet)), _p(sloc), sloc.size // 4, _p(rloc),
                                     rloc.size // 2, _p(_f32(taper))))
    return out


def modeling_f(ctx, g: Geom2d, c11, c13, c33, wavelet, slocxz, taper):
    """modeling_f (lib/vti-fwi-2d/modeling_f.cu:10): sigma_h snapshots."""
    ratio = int(np.round(np.float32(g.rate) / np.float32(g.dt)))
    nt_neg = int(round(abs(g.ot) / g.dt))
    rows = (g.nt - 1 - nt_neg) // ratio + 1
    nnxz = (g.nx + 2 * g.npad) * (g.nz + 2 * g.npad)
    out = np.zeros(max(rows, 2) * nnxz, dtype=np.float32)
    ctx.check(lib().vti2d_modeling(ctx.handle, C.byref(g), _p(_f32(c11)), _p(_f32(c13)),
                                   _p(_f32(c33)), _p(_f32(wavelet)), int(slocxz),
                                   _p(_f32(taper)), _p(out)))
    return out.reshape(-1, nnxz)


# ------------------------------------------------------------- host glue
def get_boundary(v, nx, ny, nz, npad):
    v = _f32(v)
    nb = nx * ny * nz - (nx - 2 * npad) * (ny - 2 * npad) * (nz - 2 * npad)
    out = np.empty(nb, dtype=np.float32)
    lib().vti3d_get_boundary(_p(out), _p(v), nx, ny, nz, npad)
    return out


def put_boundary(b, v, nx, ny, nz, npad):
    v = np.array(v, dtype=np.float32, copy=True)
    lib().vti3d_put_boundary(_p(_f32(b)), _p(v), nx, ny, nz, npad)
    return v


def zero_boundary(v, nx, ny, nz, npad):
    v = np.array(v, dtype=np.float32, copy=True)
    lib().vti3d_zero_boundary(_p(v), nx, ny, nz, npad)
    return v


def vepsdel_to_cij(v, eps, dl, v0=1.0, eps0=1.0, del0=1.0):
    v, eps, dl = _f32(v), _f32(eps), _f32(dl)
    c11, c13, c33 = (np.empty_like(v) for _ in range(3))
    lib().vti_vepsdel_to_cij(_p(c11), _p(c13), _p(c33), _p(v), _p(eps), _p(dl), v0, eps0, del0,
                             v.size)
    return c11, c13, c33


def grad_cij_to_vepsdel(gc11, gc13, gc33, v, eps, dl, v0=1.0, eps0=1.0, del0=1.0):
    args = [_f32(a) for a in (gc11, gc13, gc33, v, eps, dl)]
    gv, ge, gd = (np.empty_like(args[0]) for _ in range(3))
    lib().vti_grad_cij_to_vepsdel(_p(gv), _p(ge), _p(gd), *[_p(a) for a in args], v0, eps0,
                                  del0, args[0].size)
    return gv, ge, gd


def cfl_number(g: Geom3d, c11, c13, c33):
    return lib().vti3d_cfl_number(C.byref(g), _p(_f32(c11)), _p(_f32(c13)), _p(_f32(c33)))


def cfl_number2d(g: Geom2d, c11, c13, c33):
    """vti2d_cfl_number: dt^2 lambda_max of a 2D model on its padded grid."""
    return lib().vti2d_cfl_number(C.byref(g), _p(_f32(c11)), _p(_f32(c13)), _p(_f32(c33)))


def random_boundary_ref(v, n1, n2, n3, pad, pct_g=0.9, seed=2017, bval=1.0, eval_=0.2):
    """vti_random_boundary: the reference generator's random boundary of v
    (randomB.x defaults bval=1, eval=0.2); returns a new array."""
    out = np.array(v, dtype=np.float32, copy=True).reshape(-1)
    st = lib().vti_random_boundary(_p(out), n1, n2, n3, pad, pct_g, seed, bval, eval_)
    if st != VTI_OK:
        raise VtiError(st, "vti_random_boundary: invalid arguments")
    return out


def init_taper2d(nx, nz, npad):
    out = np.empty((nz + 2 * npad) * (nx + 2 * npad), dtype=np.float32)
    lib().vti2d_init_taper(_p(out), nx, nz, npad)
    return out
