#!/usr/bin/env python3
"""Generate the golden fixtures of tests/golden/ from the reference's own code.

  python tests/golden/make_golden.py --host   # here: the reference compiled for the host
                                              # (oracle/_ref/libqcs_ref_host.so)
  python tests/golden/make_golden.py --gpu    # on a B200: the reference's CUDA built for sm_100a
                                              # (oracle/_ref/libqcs_ref_gpu.so); --out DIR to
                                              # write elsewhere, then copy into tests/golden/

Each fixture (.npz) holds its seeded inputs (records, WLE rows, frames, rows)
and the parameter struct as raw bytes next to the reference's outputs, so the
tests read inputs and expected outputs from the file alone, on machines where
the reference cannot be built.  ref_host_*.npz: outputs of the host build (the
CPU oracle must equal them bit for bit); ref_gpu_*.npz: outputs of the CUDA
build (the product kernels must equal them bit for bit where the tests say so).
"""
import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "qc-storm_b200"))

import oracle_lib as O  # noqa: E402
from qcstorm_b200 import synth  # noqa: E402
from render_rows import render_para, render_rows  # noqa: E402


def para_bytes(p):
    return np.frombuffer(bytes(p), np.uint8).copy()


OUT = HERE
ONLY = None


def save(name, **arrays):
    if ONLY and not name.startswith(ONLY):
        return
    path = os.path.join(OUT, name + ".npz")
    np.savez_compressed(path, **arrays)
    print("wrote", path, os.path.getsize(path), "bytes")


def cases():
    """(name, records, para) of the localization fixtures."""
    out = []
    rec, p, _ = synth.gs2d_rois(512, R=7, seed=601)
    out.append(("gs2d7", rec, p))
    rec, p, _ = synth.as3d_rois(384, R=7, seed=602)
    out.append(("as3d7", rec, p))
    rec, p, _ = synth.multi_rois(256, R=11, seed=603)
    p.MultiEmitterFitEn = 1
    out.append(("multi11", rec, p))
    return out


def ontime_cases():
    """On-time ratios: those of the reference's consecutive-frame merge over
    blinking rows (one per call), noisy exponential decays, and edge cases (no
    molecule, small or negative first ratios, ratios above 1, NaN from an empty
    merge)."""
    out = []
    from qcstorm_b200.abi import default_para
    for loc_type in (0, 1):
        rows, counts = synth.blinking_rows(n_emitters=400, frames=24, seed=611 + loc_type, loc_type=loc_type)
        para = default_para(LocType=loc_type, ConsecFit_DistanceTh_nm=80.0, PixelSize=100.0, QE=0.8)
        _, on = O.consec(para, rows, synth.group_sizes(counts, 4), lib="ref")
        out.extend(on)
    rng = np.random.default_rng(612)
    for k in range(48):
        a, b = rng.uniform(0.2, 0.9), -rng.uniform(0.1, 3.0)
        y = a * np.exp(b * np.arange(10)) * (1 + rng.normal(0, 0.1, 10))
        out.append(y / y.sum() if k % 2 else y)
    out += [np.zeros(10), np.r_[0.005, 0.5, np.zeros(8)], np.r_[0.5, 0.005, np.zeros(8)],
            np.r_[1.2, 0.3, 0.1, np.zeros(7)], np.full(10, np.nan), np.r_[-0.1, 0.5, np.ones(8)],
            np.r_[3.0, 2.0, np.ones(8)]]
    return np.asarray(out, np.float32)


def host():
    if O.ref_host() is None:
        sys.exit("oracle/_ref/libqcs_ref_host.so not built")
    r = ontime_cases()
    mean, shown = O.ontime(r, lib="ref")
    save("ref_host_ontime", ratios=r, mean=mean, shown=shown)
    for name, rec, p in cases():
        wl = O.wle(p, rec, lib="ref")
        rows, ratios = O.localize(p, rec, wl, lib="ref")
        save("ref_host_localize_" + name, para=para_bytes(p), rois=rec, wle=wl, rows=rows, ratios=ratios)
        if name == "gs2d7":
            first, end = int(rows[:, 11].min()), int(rows[:, 11].max())
            kept = O.zero_remove(rows, 1, first, end, lib="ref")
            save("ref_host_zero_remove_gs2d7", rows=rows, first=np.int32(first), end=np.int32(end), kept=kept)
    # AS3D 9x9 at the kernel level: the reference's dispatcher sends this size to
    # its 8x8 kernel (bfgsMLE_Single_Emitter_Fit.cu:96); the true-size kernel here
    rec, p, _ = synth.as3d_rois(384, R=9, seed=602)
    wl = O.wle(p, rec, lib="ref")
    fit = O.fit_single(1, p, rec, wl, lib="ref")
    save("ref_host_fit_as3d9", para=para_bytes(p), rois=rec, wle=wl, fit=fit)
    fr, p, _ = synth.frames(3, width=128, height=96, density=60, seed=604)
    batch = 1
    ro, wo, f0, f1 = O.extract(p, fr, batch, lib="ref")
    save("ref_host_extract", para=para_bytes(p), frames=fr, batch=np.int32(batch), rois=ro, wle=wo,
         first=np.int32(f0), end=np.int32(f1))
    for loc_type in (0, 1):
        rp = render_para(loc_type, width=32, high=24, zoom=4.0)
        rows = render_rows(600, rp, seed=605 + loc_type)
        shape = (rp.SRImageHigh, rp.SRImageWidth)
        start = (np.zeros(shape, np.float32), np.zeros(shape, np.float32), 1000, np.zeros(400, np.int32))
        img, cmap, mx, hist = O.render(rp, rows, 0, state=start, lib="ref")
        save("ref_host_render_%s" % ("2d" if loc_type == 0 else "3d"), para=para_bytes(rp), rows=rows,
             start_max=np.int32(1000), image=img, colormap=cmap, max=np.int32(mx), hist=hist)


def gpu():
    if O.ref_gpu() is None:
        sys.exit("oracle/_ref/libqcs_ref_gpu.so not built")
    gpu_cases = [c for c in cases() if c[0] != "as3d7"]
    rec, p, _ = synth.as3d_rois(384, R=9, seed=602)
    gpu_cases.append(("as3d9", rec, p))
    for name, rec, p in gpu_cases:
        wl = O.ref_gpu_wle(p, rec)
        if name == "multi11":
            rows, ratios = O.ref_gpu_localize(p, rec, wl)
            save("ref_gpu_localize_" + name, para=para_bytes(p), rois=rec, wle=wl, rows=rows, ratios=ratios)
            continue
        kind = 0 if name == "gs2d7" else 1
        fit, _ = O.ref_gpu_fit_kernel(kind, p, rec, wl)
        crlb = O.ref_gpu_crlb(p, fit) if kind == 0 else None
        arrays = dict(para=para_bytes(p), rois=rec, wle=wl, fit=fit)
        if crlb is not None:
            arrays["crlb"] = crlb
        save("ref_gpu_fit_" + name, **arrays)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--host", action="store_true")
    ap.add_argument("--gpu", action="store_true")
    ap.add_argument("--out", default=HERE, help="directory for the fixtures (default: tests/golden)")
    ap.add_argument("--only", default=None, help="write only the fixtures whose name starts with this")
    a = ap.parse_args()
    OUT = a.out
    ONLY = a.only
    os.makedirs(OUT, exist_ok=True)
    if a.host:
        host()
    if a.gpu:
        gpu()
