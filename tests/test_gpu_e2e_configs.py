"""End-to-end parity of the product's own pipeline on the astigmatic 9x9 and
the 1-3 emitter 11x11 workloads, at 100,000 records per call.

Every other reference-parity test feeds one set of WLE rows to both sides.
Here each side runs its own whole call: the product's WLE pre-pass -> fit
cascade -> CRLB (qcs_loc_bfgs_mle_localization), against
  * the reference's CUDA build: its own WLE pre-pass, then for AS3D 9x9 its
    bfgsMLELoc_AS3D<9,6> kernel and CRLB (its own dispatcher would run the
    8x8 kernel, bfgsMLE_Single_Emitter_Fit.cu:96), for 11x11 its whole
    BFGS_MLELocalization (bfgs_top.cu:26-204);
  * the reference's host build, the same calls on the CPU;
  * the FP64 oracle of the same schedule, fed the product's WLE rows.
The product's WLE y widths at ROISize >= 9 follow the reference's host
build, not its CUDA build (whose nvcc-optimised spline differs by up to
100%), so rows differ from the CUDA build wherever those widths change the
weight mask or the starting width.  The rates asserted here are the measured
ones with a margin; the measured values are stated in DESIGN.md.

Reported per comparison: the decision agreement (rows per record: 0, 1 or 2
localizations), the fraction of rows accepted by both sides that fall
outside |dx|, |dy| <= 1e-3 px or relative total photons / background
<= 1e-4, and the bit-equal fraction.  Run as a script, the module prints the
full report as JSON.
"""
import json
import threading

import numpy as np
import pytest

import oracle_lib as O
from qcstorm_b200 import lib as qlib
from qcstorm_b200 import synth

N = 100_000  # records per call (<= the reference's MaxPointNum, 102,400)
CHUNKS = 16  # host-build calls in parallel threads (ctypes releases the GIL)


def per_record(rows, n, first_frame=1):
    """Rows of one call regrouped by record: the record's own row (index i)
    and the appended second-emitter row of the same frame, if any; the
    number of localizations per record (0, 1 or 2)."""
    own = rows[:n]
    extra = rows[n:]
    count = (own[:, 0] > 0).astype(np.int64)
    second = np.zeros_like(own)
    if extra.shape[0]:
        rec = extra[:, 11].astype(np.int64) - first_frame
        assert np.all((rec >= 0) & (rec < n))
        assert np.unique(rec).size == rec.size  # at most one appended row per record
        second[rec] = extra
        count[rec] += 1
    return own, second, count


def row_diffs(a, b):
    """Rows accepted by both: the fraction outside the parity tolerance and
    the fraction equal in every bit."""
    both = (a[:, 0] > 0) & (b[:, 0] > 0)
    x, y = a[both], b[both]
    dx = np.abs(x[:, 1] - y[:, 1])
    dy = np.abs(x[:, 2] - y[:, 2])
    rp = np.abs(x[:, 6] - y[:, 6]) / np.maximum(np.abs(y[:, 6]), 1e-30)
    rb = np.abs(x[:, 7] - y[:, 7]) / np.maximum(np.abs(y[:, 7]), 1e-30)
    out = (dx > 1e-3) | (dy > 1e-3) | (rp > 1e-4) | (rb > 1e-4)
    same = (x.view(np.uint32) == y.view(np.uint32)).all(axis=1)
    k = max(int(both.sum()), 1)
    return {"compared": int(both.sum()), "outside_tolerance": float(out.sum() / k),
            "bit_equal": float(same.sum() / k),
            "median_dxy_px": float(np.median(np.maximum(dx, dy))) if both.any() else 0.0,
            "p99_dxy_px": float(np.percentile(np.maximum(dx, dy), 99)) if both.any() else 0.0}


def compare_calls(rows_a, rows_b, n):
    a1, a2, ca = per_record(rows_a, n)
    b1, b2, cb = per_record(rows_b, n)
    r = {"decision_agreement": float(np.mean(ca == cb)), "first": row_diffs(a1, b1)}
    if (ca == 2).any() or (cb == 2).any():
        r["second"] = row_diffs(a2, b2)
    return r


def column_error(rows, ref64, n):
    """Each column's error of the product's rows against the FP64 oracle on
    the records both accept (positions absolute in px, the rest relative)."""
    a, _, _ = per_record(rows, n)
    b, _, _ = per_record(ref64, n)
    both = (a[:, 0] > 0) & (b[:, 0] > 0)
    names = ["peak_photons", "x", "y", "z", "sigma_x", "sigma_y", "total_photons", "background", "snr",
             "crlb_x", "crlb_y"]
    out = {"compared": int(both.sum()), "decision_agreement": float(np.mean((a[:, 0] > 0) == (b[:, 0] > 0)))}
    for c, name in enumerate(names):
        d = np.abs(a[both, c].astype(np.float64) - b[both, c])
        if name not in ("x", "y", "z"):
            d = d / np.maximum(np.abs(b[both, c].astype(np.float64)), 1e-30)
        fin = np.isfinite(d)  # AS3D CRLB: a few strongly elongated fits have none (the reference's too)
        out[name] = {"median": float(np.median(d[fin])), "p99": float(np.percentile(d[fin], 99)),
                     "not_finite": int((~fin).sum())} if fin.any() else None
    return out


def _threaded(fn, rec, *args):
    """fn over CHUNKS slices of the records in parallel host threads (each
    record has its own frame, so the WLE pre-pass is the same per slice)."""
    parts = np.array_split(np.arange(rec.shape[0]), CHUNKS)
    res = [None] * CHUNKS

    def work(i):
        res[i] = fn(rec[parts[i]], *args)

    ths = [threading.Thread(target=work, args=(i,)) for i in range(CHUNKS)]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    return parts, res


def host_fit_as3d(para, rec):
    def one(r):
        w = O.wle(para, r, "ref")
        return O.crlb(para, O.fit_single(1, para, r, w, lib="ref"), lib="ref")
    _, res = _threaded(one, rec)
    return np.concatenate(res)


def host_localize(para, rec):
    """The host build's whole localization call per slice; appended rows of
    the slices gathered after all slices' own rows (frames identify them)."""
    def one(r):
        w = O.wle(para, r, "ref")
        rows, _ = O.localize(para, r, w, lib="ref")
        return rows
    parts, res = _threaded(one, rec)
    own = np.concatenate([x[:len(p)] for x, p in zip(res, parts)])
    extra = np.concatenate([x[len(p):] for x, p in zip(res, parts)])
    return np.concatenate([own, extra])


def config_as3d9():
    rec, para, truth = synth.as3d_rois(N, R=9, seed=2401)
    ctx = qlib.LocContext(para, capacity=N)
    ours, _ = ctx.localize(rec)  # the product's WLE -> fit -> CRLB
    wl_ours = ctx.wle(rec)
    ctx.close()
    wl_ref = O.ref_gpu_wle(para, rec)
    fit_ref, _ = O.ref_gpu_fit_kernel(1, para, rec, wl_ref)
    cuda = O.ref_gpu_crlb(para, fit_ref)
    host = host_fit_as3d(para, rec)
    d64 = O.crlb(para, O.fit_single(1, para, rec, wl_ours, precision="f64"))
    return {"workload": "AS3D 9x9, %d records" % N,
            "vs_reference_cuda": compare_calls(ours, cuda, N),
            "vs_reference_host": compare_calls(ours, host, N),
            "reference_cuda_vs_host": compare_calls(cuda, host, N),
            "vs_fp64_oracle": column_error(ours, d64, N)}


def cuda_localize(para, rec, parts=2):
    """The reference CUDA build's whole call in slices of at most
    MaxPointNum / 2 = 51,200 records (the most its buffers hold with room
    for appended emitters), own rows first, then the appended ones."""
    own, extra = [], []
    for idx in np.array_split(np.arange(rec.shape[0]), parts):
        r = rec[idx]
        rows, _ = O.ref_gpu_localize(para, r, O.ref_gpu_wle(para, r))
        own.append(rows[:len(idx)])
        extra.append(rows[len(idx):])
    return np.concatenate(own + extra)


def config_multi11():
    rec, para, truth = synth.multi_rois(N, R=11, seed=2402)
    ctx = qlib.LocContext(para, capacity=N)
    ours, _ = ctx.localize(rec)
    wl_ours = ctx.wle(rec)
    ctx.close()
    cuda = cuda_localize(para, rec)
    host = host_localize(para, rec)
    d64, _ = O.localize(para, rec, wl_ours, precision="f64")
    _, _, count = per_record(ours, N)
    conf = np.zeros((3, 3), np.int64)  # true emitters 1..3 x localizations 0..2
    np.add.at(conf, (truth["k"] - 1, count), 1)
    return {"workload": "1-3 emitter 11x11, multi-emitter fitting on, %d records" % N,
            "vs_reference_cuda": compare_calls(ours, cuda, N),
            "vs_reference_host": compare_calls(ours, host, N),
            "reference_cuda_vs_host": compare_calls(cuda, host, N),
            "vs_fp64_oracle": column_error(ours, d64, N),
            "emitters_vs_localizations": conf.tolist()}


@pytest.fixture(scope="module")
def reports(cuda_ok):
    if O.ref_gpu() is None or O.ref_host() is None:
        pytest.skip("reference builds not present")
    return {"as3d9": config_as3d9(), "multi11": config_multi11()}


@pytest.mark.gpu
def test_as3d9_end_to_end(reports):
    r = reports["as3d9"]
    cuda, host, spread = r["vs_reference_cuda"], r["vs_reference_host"], r["reference_cuda_vs_host"]
    # measured: 0.9857 / 0.9972 / 0.9978 (the reference's CUDA and host builds: 0.9858)
    assert cuda["decision_agreement"] >= 0.98
    assert cuda["decision_agreement"] >= spread["decision_agreement"] - 0.003
    assert host["decision_agreement"] >= 0.995
    # rows outside the 1e-3 px / 1e-4 tolerance: no more than the two reference builds differ by
    assert cuda["first"]["outside_tolerance"] <= spread["first"]["outside_tolerance"] + 0.02
    assert host["first"]["outside_tolerance"] <= spread["first"]["outside_tolerance"] + 0.02
    f = r["vs_fp64_oracle"]
    assert f["decision_agreement"] >= 0.995
    assert f["x"]["median"] < 1e-3 and f["y"]["median"] < 1e-3
    assert f["x"]["p99"] < 0.05 and f["y"]["p99"] < 0.05


@pytest.mark.gpu
def test_multi11_end_to_end(reports):
    r = reports["multi11"]
    cuda, host, spread = r["vs_reference_cuda"], r["vs_reference_host"], r["reference_cuda_vs_host"]
    # measured: 0.9926 / 0.9989 (the reference's builds: 0.9919)
    assert cuda["decision_agreement"] >= 0.99
    assert host["decision_agreement"] >= 0.997
    assert cuda["first"]["outside_tolerance"] <= spread["first"]["outside_tolerance"] + 0.02
    # the two-emitter fit's mask has a fixed width (no WLE widths): its appended rows are the
    # reference CUDA build's bit for bit wherever both keep a second emitter
    assert cuda["second"]["compared"] > 500 and cuda["second"]["bit_equal"] >= 0.99
    f = r["vs_fp64_oracle"]
    assert f["decision_agreement"] >= 0.999
    assert f["x"]["median"] < 1e-3 and f["x"]["p99"] < 0.05


if __name__ == "__main__":
    import torch
    assert torch.cuda.is_available()
    print(json.dumps({"as3d9": config_as3d9(), "multi11": config_multi11()}, indent=1))
