"""Generate the golden fixtures by running the reference's own GPU code.

Runs oracle/_ref/ref3d and oracle/_ref/ref2d (the unmodified reference
sources compiled for sm_100a by oracle/build_ref.sh) on the seeded inputs of
cases.py and stores their outputs, with input checksums, as
tests/golden/<case>.npz. Needs a GPU; run from the repository root:

    python tests/golden/make_golden.py [--out tests/golden]
"""
from __future__ import annotations

import argparse
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
import cases as K  # noqa: E402

REF = K.ROOT / "oracle" / "_ref"


def run(binary, d, mode, *params):
    r = subprocess.run([str(REF / binary), str(d), mode, *params], capture_output=True,
                       text=True, timeout=600)
    if r.returncode != 0:
        sys.stderr.write(r.stdout[-2000:] + r.stderr[-2000:])
        raise SystemExit(f"{binary} {mode} failed with {r.returncode}")


def write_inputs3d(c, d: Path):
    """Case directory read by the harness oracle/ref_driver3d.cpp."""
    s = c["s"]
    g = s.geom()
    ns = s.souloc.size // 5
    nrec = s.recloc.size // 4
    (d / "params.txt").write_text(
        f"{s.nx} {s.ny} {s.nz} {s.nt} {s.npad} {g.ox!r} {g.oy!r} {g.oz!r} {g.ot!r} "
        f"{g.dx!r} {g.dy!r} {g.dz!r} {g.dt!r} {g.sampling_rate!r} {ns} {nrec}\n")
    for k, a in {"souloc": s.souloc, "recloc": s.recloc, "wavelet": s.wavelet,
                 "padb": c["padb"], "randb": c["randb"]}.items():
        np.asarray(a, dtype=np.float32).tofile(d / f"{k}.bin")


def write_inputs2d(s, d: Path):
    """Case directory read by the harness oracle/ref_driver2d.cpp."""
    g = s.geom()
    (d / "params.txt").write_text(
        f"{s.nx} {s.nz} {s.nt} {s.npad} {g.dx!r} {g.dz!r} {g.dt!r} {g.rate!r} {g.ot!r} "
        f"{s.sloc.size // 4} {s.rloc.size // 2}\n")
    for k in ("c11", "c13", "c33", "taper", "wavelet"):
        np.asarray(getattr(s, k), np.float32).tofile(d / f"{k}.bin")
    np.asarray(s.sloc, np.int32).tofile(d / "sloc.bin")
    np.asarray(s.rloc, np.int32).tofile(d / "rloc.bin")


def make3d(name, out):
    c = K.case3d(name)
    s = c["s"]
    with tempfile.TemporaryDirectory() as td:
        d = Path(td)
        write_inputs3d(c, d)
        np.asarray(c["cij_true"], np.float32).tofile(d / "cij.bin")
        run("ref3d", d, "model")
        dobs = np.fromfile(d / "ref_ddata.bin", dtype=np.float32)
        dobs.tofile(d / "dobs.bin")
        np.asarray(c["cij"], np.float32).tofile(d / "cij.bin")
        run("ref3d", d, "model")
        ddata = np.fromfile(d / "ref_ddata.bin", dtype=np.float32)
        run("ref3d", d, "grad")
        fg = np.fromfile(d / "ref_fgcij.bin", dtype=np.float32)
    np.savez_compressed(out / f"{name}.npz", dobs=dobs, ddata=ddata, fgcij=fg,
                        inputs=K.digest(s.souloc, s.recloc, s.wavelet, c["cij"], c["cij_true"],
                                        c["padb"], c["randb"]))
    print(name, "dobs max", np.abs(dobs).max(), "misfit/2", fg[0])


def make2d(name, out):
    c = K.case2d(name)
    s = c["s"]
    with tempfile.TemporaryDirectory() as td:
        d = Path(td)
        write_inputs2d(s, d)
        run("ref2d", d, "synthetic")
        data = np.fromfile(d / "ref_data.bin", dtype=np.float32)
        run("ref2d", d, "modeling")
        w = np.fromfile(d / "ref_wavefield.bin", dtype=np.float32)
        # observed data from the true model, gradient at the starting model
        for k in ("c11", "c13", "c33"):
            c["true"][k].tofile(d / f"{k}.bin")
        run("ref2d", d, "synthetic")
        dobs = np.fromfile(d / "ref_data.bin", dtype=np.float32)
        dobs.tofile(d / "data.bin")
        for k in ("c11", "c13", "c33"):
            np.asarray(getattr(s, k), np.float32).tofile(d / f"{k}.bin")
            c["dc"][k].tofile(d / f"d{k}.bin")
        run("ref2d", d, "grad")
        grad = np.fromfile(d / "ref_grad.bin", dtype=np.float32)
        run("ref2d", d, "gnhess")
        gnh = np.fromfile(d / "ref_gnhess.bin", dtype=np.float32)
    nnxz = (s.nx + 2 * s.npad) * (s.nz + 2 * s.npad)
    w = w.reshape(-1, nnxz)
    keep = np.arange(0, w.shape[0], 10)
    np.savez_compressed(out / f"{name}.npz", data=data, snaps=w[keep], snap_rows=keep,
                        dobs=dobs, grad=grad, gnhess=gnh,
                        inputs=K.digest(s.c11, s.c13, s.c33, s.taper, s.wavelet, s.sloc,
                                        s.rloc, *c["true"].values(), *c["dc"].values()))
    print(name, "data max", np.abs(data).max())


def make_rtm3d(name, out):
    """rtmCij3d_f of the reference: the case's observed traces (its golden
    dobs) migrated with the starting model plus random boundary."""
    c = K.case3d(name)
    s = c["s"]
    dobs = np.load(HERE / f"{name}.npz")["dobs"]
    model = K.rtm_model3d(c)
    with tempfile.TemporaryDirectory() as td:
        d = Path(td)
        write_inputs3d(c, d)
        model.astype(np.float32).tofile(d / "cij.bin")
        dobs.astype(np.float32).tofile(d / "dobs.bin")
        run("ref3d", d, "rtm")
        image = np.fromfile(d / "ref_image.bin", dtype=np.float32)
    np.savez_compressed(out / f"{name}_rtm.npz", image=image,
                        inputs=K.digest(s.souloc, s.recloc, s.wavelet, model, dobs))
    print(name, "rtm image max", np.abs(image).max())


def make_rtm2d(name, out):
    """rtm_f of the reference: the case's observed traces (golden dobs)
    migrated with the starting model."""
    c = K.case2d(name)
    s = c["s"]
    dobs = np.load(HERE / f"{name}.npz")["dobs"]
    with tempfile.TemporaryDirectory() as td:
        d = Path(td)
        write_inputs2d(s, d)
        dobs.astype(np.float32).tofile(d / "data.bin")
        run("ref2d", d, "rtm")
        image = np.fromfile(d / "ref_rtm.bin", dtype=np.float32)
    np.savez_compressed(out / f"{name}_rtm.npz", image=image,
                        inputs=K.digest(s.c11, s.c13, s.c33, s.taper, s.wavelet, s.sloc, s.rloc,
                                        dobs))
    print(name, "rtm image max", np.abs(image).max())


def make_odcig2d(name, out):
    """odcig_f of the reference: the golden dobs migrated into x-offset gathers."""
    c = K.case2d(name)
    s = c["s"]
    nhx = K.ODCIG_CASES2D[name]
    dobs = np.load(HERE / f"{name}.npz")["dobs"]
    with tempfile.TemporaryDirectory() as td:
        d = Path(td)
        write_inputs2d(s, d)
        dobs.astype(np.float32).tofile(d / "data.bin")
        run("ref2d", d, "odcig", str(nhx))
        image = np.fromfile(d / "ref_odcig.bin", dtype=np.float32)
    np.savez_compressed(out / f"{name}_odcig.npz", image=image, nhx=nhx,
                        inputs=K.digest(s.c11, s.c13, s.c33, s.taper, s.wavelet, s.sloc, s.rloc,
                                        dobs))
    print(name, "odcig max", np.abs(image).max())


def make_wgrad3d(name, out):
    """waveletGradientCij3d_f of the reference, driven by the golden dobs."""
    c = K.case3d(name)
    s = c["s"]
    dobs = np.load(HERE / f"{name}.npz")["dobs"]
    model = K.pad_model3d(c)
    with tempfile.TemporaryDirectory() as td:
        d = Path(td)
        write_inputs3d(c, d)
        model.astype(np.float32).tofile(d / "cij.bin")
        dobs.astype(np.float32).tofile(d / "dobs.bin")
        run("ref3d", d, "wgrad")
        gw = np.fromfile(d / "ref_wgrad.bin", dtype=np.float32)
    np.savez_compressed(out / f"{name}_wgrad.npz", gwavelet=gw,
                        inputs=K.digest(s.souloc, s.recloc, model, dobs))
    print(name, "wavelet gradient max", np.abs(gw).max())


def make_wgrad2d(name, out):
    """waveletGradient_f of the reference, driven by the golden dobs."""
    c = K.case2d(name)
    s = c["s"]
    dobs = np.load(HERE / f"{name}.npz")["dobs"]
    with tempfile.TemporaryDirectory() as td:
        d = Path(td)
        write_inputs2d(s, d)
        dobs.astype(np.float32).tofile(d / "data.bin")
        run("ref2d", d, "wgrad")
        gw = np.fromfile(d / "ref_wgrad.bin", dtype=np.float32)
    np.savez_compressed(out / f"{name}_wgrad.npz", gwavelet=gw,
                        inputs=K.digest(s.c11, s.c13, s.c33, s.taper, s.sloc, s.rloc, dobs))
    print(name, "wavelet gradient max", np.abs(gw).max())


def make_misfit3d(name, out):
    """objFuncGradientCij3d_f of the reference with the tpow / AGC options."""
    c = K.case3d(name)
    s = c["s"]
    dobs = np.load(HERE / f"{name}.npz")["dobs"]
    res = {}
    with tempfile.TemporaryDirectory() as td:
        d = Path(td)
        write_inputs3d(c, d)
        dobs.astype(np.float32).tofile(d / "dobs.bin")
        for key, opt in K.MISFIT_OPTIONS.items():
            np.asarray(c["cij"], np.float32).tofile(d / "cij.bin")
            run("ref3d", d, "grad", *[f"{k}={v}" for k, v in opt.items()])
            res[f"fgcij_{key}"] = np.fromfile(d / "ref_fgcij.bin", dtype=np.float32)
    np.savez_compressed(out / f"{name}_misfit.npz", **res,
                        inputs=K.digest(s.souloc, s.recloc, s.wavelet, c["cij"], c["padb"],
                                        c["randb"], dobs))
    print(name, {k: float(v[0]) for k, v in res.items()})


def make_randb(name, out):
    """The reference's random-boundary generator (oracle/_ref/ref_randb, host
    code; no GPU needed) on a seeded field."""
    n1, n2, n3, pad, pct, seed = K.RANDB_CASES[name]
    v = K.randb_input(name)
    with tempfile.TemporaryDirectory() as td:
        fi, fo = Path(td) / "in.f32", Path(td) / "out.f32"
        v.tofile(fi)
        r = subprocess.run([str(REF / "ref_randb"), str(fi), str(fo), str(n1), str(n2), str(n3),
                            str(pad), str(pct), str(seed)], capture_output=True, text=True,
                           timeout=600)
        if r.returncode != 0:
            raise RuntimeError(r.stderr)
        w = np.fromfile(fo, dtype=np.float32)
    np.savez_compressed(out / f"{name}.npz", field=w, input_digest=K.digest(v))
    print("wrote", name)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(HERE))
    ap.add_argument("--only", choices=["all", "rtm", "wgrad", "misfit", "odcig", "randb"],
                    default="all",
                    help="rtm / wgrad: only those fixtures (needs the case fixtures)")
    a = ap.parse_args()
    out = Path(a.out)
    out.mkdir(parents=True, exist_ok=True)
    if a.only == "all":
        for n in K.CASES3D:
            make3d(n, out)
        for n in K.CASES2D:
            make2d(n, out)
    if a.only in ("all", "rtm"):
        for n in K.RTM_CASES3D:
            make_rtm3d(n, out)
        for n in K.RTM_CASES2D:
            make_rtm2d(n, out)
    if a.only in ("all", "odcig"):
        for n in K.ODCIG_CASES2D:
            make_odcig2d(n, out)
    if a.only in ("all", "misfit"):
        for n in K.MISFIT_CASES3D:
            make_misfit3d(n, out)
    if a.only in ("all", "randb"):
        for n in K.RANDB_CASES:
            make_randb(n, out)
    if a.only in ("all", "wgrad"):
        for n in K.WGRAD_CASES3D:
            make_wgrad3d(n, out)
        for n in K.WGRAD_CASES2D:
            make_wgrad2d(n, out)


if __name__ == "__main__":
    main()
