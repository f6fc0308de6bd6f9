"""Test-side binding of the CPU oracle (oracle/liboracle.so) and of the host
build of the reference (oracle/_ref/libqcs_ref_host.so, present only where the
reference tree was available at build time).  Checkers only."""
import ctypes as C
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libqcs_ref_host.so")

_lib = {}


def _load(path):
    if path not in _lib:
        _lib[path] = C.CDLL(path) if os.path.exists(path) else None
    return _lib[path]


def oracle():
    lib = _load(ORACLE_SO)
    if lib is None:
        raise RuntimeError("oracle/liboracle.so not built (make -C oracle)")
    return lib


def ref_host():
    return _load(REF_SO)


def _p(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


def wle(para, rec, lib="oracle"):
    n = rec.shape[0]
    out = np.zeros((n, 6), np.float32)
    L = oracle() if lib == "oracle" else ref_host()
    f = L.qcso_wle if lib == "oracle" else L.qcsref_wle
    st = f(C.byref(para), _p(rec), n, _p(out))
    assert st == 0, st
    return out


def localize(para, rec, wl, lib="oracle", precision="f32", out_cap=None):
    n = rec.shape[0]
    cap = out_cap or max(2 * n, 1)
    out = np.zeros((cap, 12), np.float32)
    nv = C.c_int(0)
    ratios = np.zeros(7, np.float32)
    if lib == "oracle":
        f = getattr(oracle(), "qcso_localize_" + precision)
    else:
        f = ref_host().qcsref_localize
    st = f(C.byref(para), _p(rec), _p(wl), n, _p(out), cap, C.byref(nv), _p(ratios))
    assert st == 0, st
    return out[:nv.value].copy(), ratios


def fit_single(kind, para, rec, wl, lib="oracle", precision="f32"):
    n = rec.shape[0]
    out = np.zeros((n, 12), np.float32)
    if lib == "oracle":
        st = getattr(oracle(), "qcso_fit_single_" + precision)(kind, C.byref(para), _p(rec), _p(wl), n, _p(out))
    else:
        st = ref_host().qcsref_fit_kernel(kind, C.byref(para), _p(rec), _p(wl), n, _p(out))
    assert st == 0, st
    return out


def crlb(para, loc, lib="oracle"):
    out = np.ascontiguousarray(loc, np.float32).copy()
    f = oracle().qcso_crlb if lib == "oracle" else ref_host().qcsref_crlb
    st = f(C.byref(para), _p(out), out.shape[0])
    assert st == 0, st
    return out


FISHER_COLS = 8


def crlb_fisher(para, rows, rois=None):
    """The FP64 Fisher-matrix CRLB oracle (qcso_crlb_fisher_f64): n x 8."""
    rows = np.ascontiguousarray(rows, np.float32)
    n = rows.shape[0]
    out = np.zeros((max(n, 1), FISHER_COLS), np.float32)
    r = np.ascontiguousarray(rois, np.uint16) if rois is not None else None
    st = oracle().qcso_crlb_fisher_f64(C.byref(para), _p(rows), n, _p(r), r.shape[0] if r is not None else 0,
                                       _p(out))
    assert st == 0, st
    return out[:n]


EXTRACT_FMA_CONV = 1
EXTRACT_EXACT_VARIANCE = 2


def extract(para, frames, batch, start_frame=0, flags=0, lib="oracle", cap=None):
    """ROI extraction over a stack of frames fed `batch` frames per call.

    Returns (records n x R(R+1) uint16, wle n x 6, first_frame, end_frame).
    lib: "oracle" (flags select its arithmetic), "ref" (host build of the
    reference) or "ref_gpu" (the reference's CUDA build)."""
    frames = np.ascontiguousarray(frames, np.uint16)
    nf = frames.shape[0]
    R = para.ROISize
    cap = cap or 200000
    rois = np.zeros((cap, R * (R + 1)), np.uint16)
    wl = np.zeros((cap, 6), np.float32)
    n, f0, f1 = C.c_int(0), C.c_int(0), C.c_int(0)
    if lib == "oracle":
        st = oracle().qcso_extract(C.byref(para), _p(frames), nf, batch, start_frame, flags, _p(rois), _p(wl), cap,
                                   C.byref(n), C.byref(f0), C.byref(f1))
    else:
        L = ref_host() if lib == "ref" else ref_gpu()
        f = L.qcsref_extract if lib == "ref" else L.qcsrefg_extract
        st = f(C.byref(para), _p(frames), nf, batch, start_frame, _p(rois), _p(wl), cap, C.byref(n), C.byref(f0),
               C.byref(f1))
    assert st == 0, st
    k = min(n.value, cap)
    return rois[:k].copy(), wl[:k].copy(), f0.value, f1.value


def set_threads(n):
    oracle().qcso_set_threads(int(n))


REF_GPU_SO = os.path.join(ROOT, "oracle", "_ref", "libqcs_ref_gpu.so")


def ref_gpu():
    """The reference CUDA library built for sm_100a (checker on GPU hosts)."""
    return _load(REF_GPU_SO)


def ref_gpu_fit_kernel(kind, para, rec, wl):
    n = rec.shape[0]
    out = np.zeros((n, 12), np.float32)
    ms = C.c_float(0)
    st = ref_gpu().qcsrefg_fit_kernel(kind, C.byref(para), _p(rec), _p(wl), n, _p(out), C.byref(ms))
    assert st == 0, st
    return out, ms.value


def ref_gpu_localize(para, rec, wl):
    n = rec.shape[0]
    cap = max(2 * n, 1)
    out = np.zeros((cap, 12), np.float32)
    nv = C.c_int(0)
    ratios = np.zeros(7, np.float32)
    st = ref_gpu().qcsrefg_localize(C.byref(para), _p(rec), _p(wl), n, _p(out), cap, C.byref(nv), _p(ratios))
    assert st == 0, st
    return out[:nv.value].copy(), ratios


def ref_gpu_wle(para, rec):
    out = np.zeros((rec.shape[0], 6), np.float32)
    st = ref_gpu().qcsrefg_wle(C.byref(para), _p(rec), rec.shape[0], _p(out))
    assert st == 0, st
    return out


def ref_gpu_crlb(para, loc):
    out = np.ascontiguousarray(loc, np.float32).copy()
    st = ref_gpu().qcsrefg_crlb(C.byref(para), _p(out), out.shape[0])
    assert st == 0, st
    return out


def zero_remove(rows, sort_frame=0, first_frame=0, end_frame=0, lib="oracle"):
    """RemoveZeroLocalizations through the oracle ("oracle"), the host build
    ("ref") or the reference's CUDA build ("ref_gpu")."""
    rows = np.ascontiguousarray(rows, np.float32)
    out = np.zeros_like(rows)
    n = C.c_int(0)
    if lib == "oracle":
        f = oracle().qcso_zero_remove
    elif lib == "ref":
        f = ref_host().qcsref_zero_remove
    else:
        f = ref_gpu().qcsrefg_zero_remove
    st = f(_p(rows), rows.shape[0], int(sort_frame), int(first_frame), int(end_frame), _p(out), C.byref(n))
    assert st == 0, st
    return out[:n.value].copy()


def consec(para, rows, sizes, is_end=None, lib="oracle", gpu_rounding=0):
    """ConsecutiveFit_WeightedAvg over groups of rows (sizes[g] rows each, in
    turn) through the oracle ("oracle"; gpu_rounding 1: the GPU's roundings),
    the host build of the reference ("ref") or its CUDA build ("ref_gpu").
    Returns (list of per-call output rows, ontime ratios [groups, 10])."""
    rows = np.ascontiguousarray(rows, np.float32)
    sizes = np.ascontiguousarray(sizes, np.int32)
    g = sizes.size
    if is_end is None:
        is_end = np.zeros(g, np.int32)
        is_end[-1] = 1
    is_end = np.ascontiguousarray(is_end, np.int32)
    out = np.zeros((max(rows.shape[0], 1), 12), np.float32)
    out_n = np.zeros(g, np.int32)
    ontime = np.zeros((g, 10), np.float32)
    pp = C.byref(para)
    if lib == "oracle":
        st = oracle().qcso_consec(pp, _p(rows), _p(sizes), _p(is_end), g, int(gpu_rounding), _p(out), _p(out_n),
                                  _p(ontime))
    elif lib == "ref":
        st = ref_host().qcsref_consec(pp, _p(rows), _p(sizes), _p(is_end), g, _p(out), _p(out_n), _p(ontime))
    else:
        st = ref_gpu().qcsrefg_consec(pp, _p(rows), _p(sizes), _p(is_end), g, _p(out), _p(out_n), _p(ontime))
    assert st == 0, st
    res, o = [], 0
    for k in out_n:
        res.append(out[o:o + k].copy())
        o += k
    return res, ontime


def stat(para, rows, sizes, lib="oracle"):
    """GetStatisticalInf over groups of rows (sizes[g] each, in turn) through the
    oracle ("oracle"), the host build of the reference ("ref") or its CUDA
    build ("ref_gpu").  Returns (histograms [groups, 4, 1600], means [groups, 10])."""
    rows = np.ascontiguousarray(rows, np.float32)
    sizes = np.ascontiguousarray(sizes, np.int32)
    g = sizes.size
    hist = np.zeros((g, 4, 1600), np.int32)
    means = np.zeros((g, 10), np.float32)
    pp = C.byref(para)
    if lib == "oracle":
        st = oracle().qcso_stat(pp, _p(rows), _p(sizes), g, _p(hist), _p(means))
    elif lib == "ref":
        st = ref_host().qcsref_stat(pp, _p(rows), _p(sizes), g, _p(hist), _p(means))
    else:
        st = ref_gpu().qcsrefg_stat(pp, _p(rows), _p(sizes), g, _p(hist), _p(means))
    assert st == 0, st
    return hist, means


def ontime(ratios, lib="oracle"):
    """UpdateOntimeRatio over calls of 10 on-time ratios each (ratios [calls, 10])
    through the oracle ("oracle") or the host build of the reference ("ref").
    Returns (mean on time [calls], shown ratios [calls, 10])."""
    ratios = np.ascontiguousarray(np.atleast_2d(ratios), np.float32)
    c = ratios.shape[0]
    mean = np.zeros(c, np.float32)
    out = np.zeros((c, 10), np.float32)
    if lib == "oracle":
        for k in range(c):
            m = C.c_float()
            st = oracle().qcso_ontime(_p(ratios[k]), 10, C.byref(m), _p(out[k]))
            assert st == 0, st
            mean[k] = m.value
    else:
        st = ref_host().qcsref_ontime(_p(ratios), c, _p(mean), _p(out))
        assert st == 0, st
    return mean, out


def render(para, rows, mode, fixed_prec=0.0, state=None, lib="oracle"):
    """Super-resolution render of rows through the oracle ("oracle"), the host
    build of the reference ("ref") or its CUDA build ("ref_gpu").  state:
    (image, colormap, max, hist) to start from (zeros when None).  Returns the
    updated (image, colormap, max, hist)."""
    rows = np.ascontiguousarray(rows, np.float32)
    shape = (para.SRImageHigh, para.SRImageWidth)
    if state is None:
        img, cmap = np.zeros(shape, np.float32), np.zeros(shape, np.float32)
        mx, hist = 0, np.zeros(400, np.int32)
    else:
        img, cmap, mx, hist = (np.array(state[0], np.float32), np.array(state[1], np.float32), int(state[2]),
                               np.array(state[3], np.int32))
    m = C.c_int(mx)
    f = {"oracle": lambda: oracle().qcso_render, "ref": lambda: ref_host().qcsref_render,
         "ref_gpu": lambda: ref_gpu().qcsrefg_render}[lib]()
    st = f(C.byref(para), _p(rows), rows.shape[0], int(mode), C.c_float(fixed_prec), _p(img), _p(cmap),
           C.byref(m), _p(hist))
    assert st == 0, st
    return img, cmap, m.value, hist
