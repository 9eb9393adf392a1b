"""CPU tests of the C-ABI library's host side: it loads, exports every symbol
its header declares, and its host glue matches the reference formulas."""
import ctypes
import re

import numpy as np
import pytest

import cases as K
from conftest import ROOT, load_golden, rel_l2

import vtib200 as V


def header_functions():
    txt = (ROOT / "include" / "vti_b200.h").read_text()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(vti\w+)\s*\(", txt)))


def test_library_loads_and_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(V.LIB_PATH))
    names = header_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_declares_only_header_symbols():
    assert set(V.exported_symbols()) <= set(header_functions())


@pytest.mark.parametrize("lang", [("gcc", "c", "-std=c99"), ("g++", "c++", "-std=c++17")])
def test_c_abi_header_is_plain_c(lang, tmp_path):
    """include/vti_b200.h compiles as strict C99 (pedantic, warnings as
    errors) and as C++: no C++ or CUDA types in the boundary."""
    import subprocess
    cc, x, std = lang
    src = tmp_path / "use.c"
    src.write_text('#include "vti_b200.h"\nint main(void) { return VTI_OK; }\n')
    r = subprocess.run([cc, std, "-Wall", "-Wextra", "-pedantic", "-Werror", "-fsyntax-only",
                        "-x", x, "-I", str(ROOT / "include"), str(src)],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr[-2000:]


@pytest.mark.parametrize("header", sorted(p.name for p in (ROOT / "include").glob("*.h")))
def test_every_header_compiles_on_its_own(header, tmp_path):
    """Each header of include/ is self-contained C++ (warnings as errors)."""
    import subprocess
    src = tmp_path / "use.cpp"
    src.write_text(f'#include "{header}"\nint main() {{ return 0; }}\n')
    r = subprocess.run(["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-fsyntax-only",
                        "-I", str(ROOT / "include"), str(src)],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr[-2000:]


@pytest.mark.parametrize("dim", ["3d", "2d"])
def test_reference_harness_links_against_the_shim(dim, tmp_path):
    """The harness that drives the reference's C++ entry points and operator
    classes (oracle/ref_driver{3d,2d}.cpp) compiles against include/ and links
    to libvti_wave.so alone: every entry it calls is exported with the
    reference's C++ signature. Nothing is run."""
    import subprocess
    libdir = V.LIB_PATH.parent
    exe = tmp_path / f"shim{dim}"
    r = subprocess.run(
        ["g++", "-O0", "-std=c++17", "-DVTI_SHIM", str(ROOT / "oracle" / f"ref_driver{dim}.cpp"),
         str(ROOT / "tests" / "shim" / "myio_stub.cpp"), "-I", str(ROOT / "include"),
         f"-L{libdir}", "-lvti_wave", "-lvti_b200", f"-Wl,-rpath,{libdir}", "-o", str(exe)],
        capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-3000:]
    assert exe.exists()


def _boundary_mask(nx, ny, nz, npad):
    m = np.ones((nz, ny, nx), dtype=bool)
    m[npad:nz - npad, npad:ny - npad, npad:nx - npad] = False
    return m.reshape(-1)


@pytest.mark.parametrize("dims", [(12, 10, 9, 2), (20, 16, 14, 4), (9, 9, 9, 1)])
def test_boundary_get_put_zero(dims):
    nx, ny, nz, npad = dims
    rng = np.random.default_rng(0)
    v = rng.standard_normal(nx * ny * nz).astype(np.float32)
    b = V.get_boundary(v, nx, ny, nz, npad)
    mask = _boundary_mask(nx, ny, nz, npad)
    assert b.size == mask.sum()
    # the list holds exactly the pad-region values, in the x-fastest scan order
    np.testing.assert_array_equal(b, v[mask])
    w = V.put_boundary(b * 2, v, nx, ny, nz, npad)
    np.testing.assert_array_equal(w[mask], 2 * v[mask])
    np.testing.assert_array_equal(w[~mask], v[~mask])
    z = V.zero_boundary(v, nx, ny, nz, npad)
    assert not z[mask].any()
    np.testing.assert_array_equal(z[~mask], v[~mask])


def test_converted_inputs_outlive_the_call():
    """Float64 inputs are converted to float32 temporaries; those must stay
    alive until the C call returns. The arrays are large enough that a freed
    temporary is returned to the system and reading it would fault."""
    nx, ny, nz, npad = 96, 96, 64, 12
    rng = np.random.default_rng(3)
    v = rng.standard_normal(nx * ny * nz).astype(np.float32)
    b64 = rng.standard_normal(int(_boundary_mask(nx, ny, nz, npad).sum()))
    w64 = V.put_boundary(b64, v, nx, ny, nz, npad)
    w32 = V.put_boundary(b64.astype(np.float32), v, nx, ny, nz, npad)
    np.testing.assert_array_equal(w64, w32)
    g = V.geom3d(nx, ny, nz, 100, npad, 10.0, 10.0, 10.0, 1e-3, 4e-3)
    c = np.full(nx * ny * nz, 4.0e6)
    assert V.cfl_number(g, c, c * 0.5, c) == V.cfl_number(g, *(x.astype(np.float32)
                                                              for x in (c, c * 0.5, c)))


def test_vepsdel_conversion_and_chain_rule():
    rng = np.random.default_rng(1)
    n = 1000
    v = rng.uniform(1.5, 4.5, n).astype(np.float32)
    eps = rng.uniform(0, 0.2, n).astype(np.float32)
    dl = rng.uniform(0, 0.1, n).astype(np.float32)
    v0, e0, d0 = 1000.0, 1.0, 1.0
    c11, c13, c33 = V.vepsdel_to_cij(v, eps, dl, v0, e0, d0)
    vv = (v0 * v.astype(np.float64)) ** 2
    np.testing.assert_allclose(c33, vv, rtol=1e-6)
    np.testing.assert_allclose(c11, vv * (1 + 2 * eps), rtol=1e-6)
    np.testing.assert_allclose(c13, vv * np.sqrt(1 + 2 * dl), rtol=1e-6)
    # chain rule = transpose of the Jacobian: <g, dC/dm dm> = <J^T g, dm>
    g = [rng.standard_normal(n).astype(np.float32) for _ in range(3)]
    gv, ge, gd = V.grad_cij_to_vepsdel(*g, v, eps, dl, v0, e0, d0)
    h = 1e-3
    for k, (gm, arr) in enumerate(zip((gv, ge, gd), (v, eps, dl))):
        dm = np.zeros((3, n), dtype=np.float64)
        dm[k] = 1.0
        args_p = [v.astype(np.float64), eps.astype(np.float64), dl.astype(np.float64)]
        args_m = [a.copy() for a in args_p]
        args_p[k] = args_p[k] + h
        args_m[k] = args_m[k] - h

        def cij(a):
            q = (v0 * a[0]) ** 2
            return q * (1 + 2 * e0 * a[1]), q * np.sqrt(1 + 2 * d0 * a[2]), q

        cp, cm = cij(args_p), cij(args_m)
        fd = sum(g[j].astype(np.float64) * (cp[j] - cm[j]) / (2 * h) for j in range(3))
        assert rel_l2(gm, fd) < 1e-4, k


def test_check_eps_del_projection():
    eps = np.array([0.1, 0.05, 0.2], dtype=np.float32)
    dl = np.array([0.05, 0.1, 0.2], dtype=np.float32)
    lib = V.lib()
    mask = np.zeros(3, dtype=np.float32)
    cnt = lib.vti_check_eps_del(V._p(eps), V._p(dl), 1.0, 1.0, 3, V._p(mask))
    assert cnt == 1
    assert eps[1] == dl[1]  # projected onto del == eps
    assert list(mask) == [0.0, 2.0, 1.0]


def test_cfl_number_matches_eigenvalues():
    rng = np.random.default_rng(2)
    n = 200
    c33 = rng.uniform(1.5e3, 4.5e3, n).astype(np.float32) ** 2
    c11 = (c33 * rng.uniform(1.0, 1.4, n)).astype(np.float32)
    c13 = (c33 * rng.uniform(1.0, 1.2, n)).astype(np.float32)
    g = V.geom3d(2, 2, n // 4, 10, 0, 10.0, 12.0, 8.0, 1e-3, 2e-3)
    g.nx, g.ny, g.nz = 2, 2, n // 4
    cfl = V.cfl_number(g, c11, c13, c33)
    C = np.array([-2.84722222222, 1.6, -0.2, 0.02539682539, -0.00178571428])
    s = abs(C[0] + 2 * sum(C[k] * (-1) ** k for k in range(1, 5)))
    kh, kz = s / 10.0**2 + s / 12.0**2, s / 8.0**2
    lam = max(np.linalg.eigvals(np.array([[a * kh, b * kz], [b * kh, c * kz]])).real.max()
              for a, b, c in zip(c11.astype(np.float64), c13.astype(np.float64),
                                 c33.astype(np.float64)))
    dt2 = float(np.float32(1e-3)) ** 2
    assert abs(cfl - lam * dt2) / (lam * dt2) < 1e-9


def test_cfl_number_2d_and_nonfinite_models():
    rng = np.random.default_rng(5)
    nx, nz, npad = 7, 5, 2
    n = (nx + 2 * npad) * (nz + 2 * npad)
    c33 = rng.uniform(1.5e3, 4.5e3, n).astype(np.float32) ** 2
    c11 = (c33 * rng.uniform(1.0, 1.4, n)).astype(np.float32)
    c13 = (c33 * rng.uniform(1.0, 1.2, n)).astype(np.float32)
    g = V.geom2d(nx, nz, 10, npad, 10.0, 8.0, 1e-3, 2e-3)
    cfl = V.cfl_number2d(g, c11, c13, c33)
    C = np.array([-2.84722222222, 1.6, -0.2, 0.02539682539, -0.00178571428])
    s = abs(C[0] + 2 * sum(C[k] * (-1) ** k for k in range(1, 5)))
    kh, kz = s / 10.0**2, s / 8.0**2
    lam = max(np.linalg.eigvals(np.array([[a * kh, b * kz], [b * kh, c * kz]])).real.max()
              for a, b, c in zip(c11.astype(np.float64), c13.astype(np.float64),
                                 c33.astype(np.float64)))
    dt2 = float(np.float32(1e-3)) ** 2
    assert abs(cfl - lam * dt2) / (lam * dt2) < 1e-9
    # a NaN anywhere in the model gives NaN (which every entry point refuses)
    c11[n // 2] = np.nan
    assert np.isnan(V.cfl_number2d(g, c11, c13, c33))
    g3 = V.geom3d(nx, nz, 1, 10, 0, 10.0, 10.0, 8.0, 1e-3, 2e-3)
    g3.nx, g3.ny, g3.nz = n, 1, 1
    assert np.isnan(V.cfl_number(g3, c11, c13, c33))


def test_taper2d_profile():
    nx, nz, npad = 20, 10, 5
    t = V.init_taper2d(nx, nz, npad).reshape(nz + 2 * npad, nx + 2 * npad)
    pi = np.float64(np.float32(4 * np.arctan(np.float32(1))))
    t0 = (np.float32(0.95) + (1 - np.float64(np.float32(0.95))) *
          np.cos(pi * (npad - 1 - np.arange(npad)) / npad)).astype(np.float32)
    assert np.all(t[npad:-npad, npad:-npad] == 1)
    np.testing.assert_allclose(t[nz // 2 + npad, :npad], t0, rtol=1e-7)
    np.testing.assert_allclose(t[nz // 2 + npad, -npad:], t0[::-1], rtol=1e-7)
    np.testing.assert_allclose(t[0, 0], t0[0] * t0[0], rtol=1e-6)


def header_prototypes():
    """name -> parameter count of every function declared in vti_b200.h."""
    txt = (ROOT / "include" / "vti_b200.h").read_text()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    out = {}
    for m in re.finditer(r"\b(vti\w+)\s*\(([^;{]*?)\)\s*;", txt, flags=re.S):
        params = m.group(2).strip()
        out[m.group(1)] = 0 if params in ("", "void") else params.count(",") + 1
    return out


def test_binding_argument_counts_match_header():
    protos = header_prototypes()
    wrong = {name: (len(args), protos[name]) for name, (_, args) in V._signatures().items()
             if name in protos and len(args) != protos[name]}
    assert not wrong, wrong


@pytest.mark.parametrize("name", sorted(K.RANDB_CASES))
def test_random_boundary_matches_reference_generator(name):
    """vti_random_boundary reproduces the reference's random-boundary
    generator (lib/random-boundary/randomBound.h:48, as randomB.x calls it)
    bit for bit: same C library rand() sequence, same cluster walk."""
    n1, n2, n3, pad, pct, seed = K.RANDB_CASES[name]
    v = K.randb_input(name)
    gold = load_golden(name)
    assert str(gold["input_digest"]) == K.digest(v)
    out = V.random_boundary_ref(v, n1, n2, n3, pad, pct, seed)
    np.testing.assert_array_equal(out, gold["field"])
    # only the pad changes, and the velocity is only lowered
    inner = V.zero_boundary(np.ones(v.size, dtype=np.float32), n1, n2, n3, pad) if n3 > 1 else None
    r = out / v
    assert r.max() <= 1.0 and r.min() > 0.2 / 3
    if inner is not None:
        assert np.all(r[inner == 1] == 1.0)


def test_oracle_host_helpers_equal_the_library():
    """The oracle's numpy restatements of getBoundary / putBoundary /
    VEpsDel2Cij give the library's arrays bit for bit, so inputs built with
    the oracle alone (the reference leg of the benchmark) are the same."""
    import oracle as O
    rng = np.random.default_rng(0)
    nx, ny, nz, npad = 23, 19, 17, 5
    n = nx * ny * nz
    v = rng.uniform(1500, 4500, n).astype(np.float32)
    e = rng.uniform(0, 0.2, n).astype(np.float32)
    d = rng.uniform(0, 0.1, n).astype(np.float32)
    for a, b in zip(O.vepsdel_to_cij(v, e, d), V.vepsdel_to_cij(v, e, d)):
        np.testing.assert_array_equal(a, b)
    for a, b in zip(O.vepsdel_to_cij(v, e, d, 1.1, 0.9, 1.3), V.vepsdel_to_cij(v, e, d, 1.1, 0.9, 1.3)):
        np.testing.assert_array_equal(a, b)
    bo, bl = O.get_boundary(v, nx, ny, nz, npad), V.get_boundary(v, nx, ny, nz, npad)
    np.testing.assert_array_equal(bo, bl)
    w = rng.uniform(0, 1, n).astype(np.float32)
    np.testing.assert_array_equal(O.put_boundary(bo, w, nx, ny, nz, npad),
                                  V.put_boundary(bl, w, nx, ny, nz, npad))


def test_gradient_inputs_built_by_the_oracle_equal_the_library_ones():
    import oracle as O
    import vtib200.synth as S
    kw = dict(S.GRADIENT400, nx=48, ny=40, nz=32, nt=50, npad=8, smooth_m=60.0)
    a = S.gradient_inputs(kw)
    b = S.gradient_inputs(kw, get_boundary=O.get_boundary, put_boundary=O.put_boundary,
                          vepsdel_to_cij=O.vepsdel_to_cij)
    for x, y in zip(a[1:], b[1:]):
        np.testing.assert_array_equal(x, y)


def test_reference_callers_link_against_the_shim():
    """The reference's own FWI and RTM executables (3D fwi3d-lbfgsc, 3D
    rtm3d-cij-shot, 2D fwi-lbfgs-c-param with its objFuncGradient.cu glue),
    compiled from the reference tree with its own headers, link against
    libvti_wave.so with none of the reference's GPU objects: the entries they
    call (objFuncGradientVEpsDel, rtmCij3d_f, objFuncGradient_f) are the
    shim's. Needs the reference tree (oracle/link_callers.sh); nothing runs."""
    import subprocess
    r = subprocess.run(["bash", str(ROOT / "oracle" / "link_callers.sh")], capture_output=True,
                       text=True, timeout=900)
    if "skipping" in r.stderr:
        pytest.skip("reference tree not present")
    assert r.returncode == 0, r.stderr[-3000:]
    out = ROOT / "oracle" / "_ref" / "callers"
    for exe in ("fwi3d-lbfgsc", "rtm3d-cij-shot", "fwi-lbfgs-c-param"):
        assert (out / exe).exists()
    shim = V.LIB_PATH.parent / "libvti_wave.so"
    exported = subprocess.run(["nm", "-D", "--defined-only", str(shim)], capture_output=True,
                              text=True).stdout
    for obj, sym in (("fwi3d-lbfgsc.cu.o", "objFuncGradientVEpsDel"),
                     ("rtm3d-cij-shot.cu.o", "rtmCij3d_f"),
                     ("objFuncGradient.cu.o", "objFuncGradient_f")):
        undef = subprocess.run(["nm", "-u", "-C", str(out / obj)], capture_output=True,
                               text=True).stdout
        assert sym in undef, (obj, sym)          # the caller needs it from outside
        assert sym in subprocess.run(["c++filt"], input=exported, capture_output=True,
                                     text=True).stdout, sym  # and the shim exports it


def _pack_f16_numpy(t, nnt):
    """The packing the library documents, restated with numpy: per time
    sample the largest |value| over all traces (1 where 0), values times the
    FP32 reciprocal of it rounded to the nearest half."""
    a = np.asarray(t, dtype=np.float32).reshape(-1, nnt)
    sc = np.abs(a).max(axis=0, initial=np.float32(0))
    sc = np.where(sc > 0, sc, np.float32(1)).astype(np.float32)
    inv = (np.float32(1) / sc).astype(np.float32)
    h = (a * inv).astype(np.float16)
    return sc, h


@pytest.mark.parametrize("nr,nnt", [(7, 33), (40, 8), (1, 1), (0, 5), (300, 751)])
def test_traces_f16_block_matches_the_documented_packing(nr, nnt):
    rng = np.random.default_rng(nr * 1000 + nnt)
    decay = np.exp(-np.arange(nnt) / max(nnt / 6, 1)).astype(np.float32)
    t = (rng.standard_normal((nr, nnt)) * decay).astype(np.float32)
    if nr > 2:
        t[:, nnt // 2] = 0.0  # an all-zero time plane packs with scale 1
    block = V.pack_traces_f16(t, nnt)
    assert block.size == V.traces_f16_bytes(nr, nnt) == 4 * nnt + 2 * nr * nnt
    sc, h = _pack_f16_numpy(t, nnt)
    np.testing.assert_array_equal(block[:4 * nnt].view(np.float32), sc)
    np.testing.assert_array_equal(block[4 * nnt:].view(np.float16).reshape(nr, nnt), h)
    back = V.unpack_traces_f16(block, nr, nnt)
    np.testing.assert_array_equal(back, (h.astype(np.float32) * sc).reshape(-1))
    if nr:
        # every sample keeps the half's relative precision against its plane
        err = np.abs(back.reshape(nr, nnt) - t) / sc
        assert err.max() <= 2.0 ** -11 * 1.0001


def test_traces_f16_packing_refuses_nonfinite_samples():
    t = np.ones((3, 5), dtype=np.float32)
    t[1, 2] = np.nan
    with pytest.raises(V.VtiError):
        V.pack_traces_f16(t, 5)
