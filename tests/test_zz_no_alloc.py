"""The allocation-free localization entry point (qcs_localize_noalloc).

It serves callers that cannot allocate device memory: code recording the
localization into a CUDA graph during stream capture (cudaMalloc is not
allowed there), hosts that own all device memory through their own pool, and
camera-rate loops that cannot take cudaMalloc's device-wide synchronisation.
Checked through the C ABI against the context-based entry point
qcs_loc_localize_device on the same device records: equal bits (the
tolerance of every GPU-to-GPU comparison in this suite), on two calls in a
row with different data (the shared scratch array keeps the first call's
contents), plus the size limit.  Collected last, so that a run stopping at the
first failure has run everything else.
"""
import ctypes as C

import numpy as np
import pytest

from qcstorm_b200 import lib as qlib
from qcstorm_b200 import synth

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


class _DeviceView:
    """A raw device pointer seen as an array (read with torch.as_tensor)."""

    def __init__(self, ptr, shape, typestr):
        self.__cuda_array_interface__ = {"shape": shape, "typestr": typestr, "data": (int(ptr), False),
                                         "version": 2}


def run_both(rec, para):
    import torch
    n = rec.shape[0]
    lib = qlib.load()
    ctx = qlib.LocContext(para, capacity=n)
    wle = ctx.wle(rec)
    s = torch.cuda.Stream()
    d_rec = torch.from_numpy(np.ascontiguousarray(rec).view(np.int16)).cuda()
    d_wle = torch.from_numpy(wle).cuda()
    torch.cuda.synchronize()
    # existing entry point: rows stay in the context's device buffer
    ctx.localize_device(d_rec.data_ptr(), n, d_wle.data_ptr(), s.cuda_stream)
    s.synchronize()
    cnt_ctx = int(torch.as_tensor(_DeviceView(lib.qcs_loc_device_valid_num(ctx.h), (1,), "<i4"),
                                  device="cuda").cpu()[0])
    rows_ctx = torch.as_tensor(_DeviceView(lib.qcs_loc_device_rows(ctx.h), (cnt_ctx, 12), "<f4"),
                               device="cuda").cpu().numpy()
    # allocation-free entry point on caller-owned buffers
    d_rows = torch.full((2 * n, 12), -1.0, dtype=torch.float32, device="cuda")
    d_cnt = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    qlib.check(lib.qcs_localize_noalloc(C.byref(para), C.c_void_p(d_rec.data_ptr()), C.c_void_p(d_wle.data_ptr()), n,
                                        C.c_void_p(d_rows.data_ptr()), C.c_void_p(d_cnt.data_ptr()),
                                        C.c_void_p(s.cuda_stream)))
    s.synchronize()
    cnt = int(d_cnt.cpu()[0])
    rows = d_rows.cpu().numpy()[:cnt]
    ctx.close()
    return cnt_ctx, rows_ctx, cnt, rows


def test_noalloc_matches_context_entry_point_twice(cuda_ok):
    first = synth.multi_rois(4000, R=7, seed=501)
    second = synth.as3d_rois(3000, R=9, seed=502)
    second[1].MultiEmitterFitEn = 1
    for rec, para, _ in (first, second):
        n_ctx, rows_ctx, n_na, rows_na = run_both(rec, para)
        assert n_na == n_ctx
        assert n_na >= rec.shape[0]
        assert np.array_equal(bits(rows_ctx), bits(rows_na))


def test_noalloc_size_limit(cuda_ok):
    _, para, _ = synth.gs2d_rois(16, R=7, seed=1)
    code = qlib.load().qcs_localize_noalloc(C.byref(para), C.c_void_p(16), C.c_void_p(16), 8193, C.c_void_p(16),
                                            None, None)
    assert code == 3  # QCS_ERR_CAPACITY, rejected before any device work


def test_noalloc_refuses_unaligned_rows(cuda_ok):
    _, para, _ = synth.gs2d_rois(16, R=7, seed=1)
    code = qlib.load().qcs_localize_noalloc(C.byref(para), C.c_void_p(16), C.c_void_p(16), 16, C.c_void_p(16 + 4),
                                            None, None)
    assert code == 1  # QCS_ERR_ARG: rows are written 16 bytes at a time; rejected before any device work


def test_noalloc_refuses_nonpositive_qe(cuda_ok):
    _, para, _ = synth.gs2d_rois(16, R=7, seed=1)
    for qe in (0.0, -0.5, float("nan")):
        para.QE = qe
        code = qlib.load().qcs_localize_noalloc(C.byref(para), C.c_void_p(16), C.c_void_p(16), 16, C.c_void_p(16),
                                                None, None)
        assert code == 1  # QCS_ERR_ARG before any device work: the CRLB divides by QE
