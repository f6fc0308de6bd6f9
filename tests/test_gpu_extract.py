"""ROI extraction on the GPU (qcs_extract_*), checked through the C ABI.

Against the oracle in its device arithmetic mode (fused-multiply-add taps,
exact-sum variance: the product's defined arithmetic) the records, their
order and the frame range are equal bit for bit.  The WLE rows of those
records are the GPU WLE pass, whose spline arithmetic follows the reference's
CUDA build (contracted multiply-adds) rather than the host-order oracle: they
are checked bit for bit against the product's own WLE entry point on the same
records and, within 1e-5 relative error and with the same
nearest-neighbour distances, against the oracle.  Against the reference's
own CUDA build (oracle/_ref/libqcs_ref_gpu.so) records and WLE rows are equal
bit for bit as sets: the reference appends records in GPU arrival order, so
both sides are sorted by (frame, y, x) first.  At ROISize >= 9 the
comparison with that build covers the nearest-neighbour distance and the x
widths only: nvcc's optimised build of the reference's spline
(WLEParaEstimation_core.h:136-147) returns y widths (sigmaU, sigmaD) that
differ from its own host build and from an unoptimised (-G) build of the
same code, by up to 100 %; the product computes what the source states.
"""
import ctypes as C
import os

import numpy as np
import pytest

import oracle_lib as O
from qcstorm_b200 import abi
from qcstorm_b200 import lib as qlib
from qcstorm_b200 import synth

pytestmark = pytest.mark.gpu

DEVICE_MODE = O.EXTRACT_FMA_CONV | O.EXTRACT_EXACT_VARIANCE

# (name, width, height, frames, batch, LocType, MultiEmitterFitEn, ROISize, density, seed)
CASES = [
    ("gs2d_multi_r7", 256, 192, 4, 2, 0, 1, 7, 150, 21),
    ("gs2d_single_r7", 256, 192, 4, 4, 0, 0, 7, 150, 22),
    ("as3d_r9_odd_width", 200, 160, 3, 1, 1, 0, 9, 100, 23),
    ("as3d_multi_r11", 288, 240, 2, 2, 1, 1, 11, 120, 24),
    ("gs2d_multi_r13_ragged", 197, 183, 3, 3, 0, 1, 13, 80, 25),
    ("gs2d_single_r5", 96, 80, 6, 3, 0, 0, 5, 30, 26),
    ("gs2d_single_r17", 256, 256, 2, 2, 0, 0, 17, 60, 27),
    ("frame_512_batch4", 512, 512, 4, 4, 0, 1, 7, 800, 28),
]


def make(case):
    name, W, H, nf, batch, lt, multi, R, dens, seed = case
    fr, para, _ = synth.frames(nf, width=W, height=H, density=dens, seed=seed)
    para.LocType, para.MultiEmitterFitEn, para.ROISize = lt, multi, R
    return fr, para, batch


def run_product(fr, para, batch, start_frame=0, source="normal", capacity=0):
    ctx = qlib.ExtractContext(para, max_batched_num=batch, capacity=capacity)
    if source == "gpu":
        import torch
        d = torch.from_numpy(fr.view(np.int16)).cuda()
        torch.cuda.synchronize()
        per = fr.shape[1] * fr.shape[2]
        for f in range(0, fr.shape[0], batch):
            nb = min(batch, fr.shape[0] - f)
            ctx.extract_device(d.data_ptr() + f * per * 2, nb, start_frame + f)
    else:
        for f in range(0, fr.shape[0], batch):
            ctx.extract(fr[f:f + batch], start_frame + f)
    rois, wle = ctx.records()
    out = rois, wle, ctx.frame_range(), ctx.dropped()
    ctx.close()
    return out


def sort_by_key(rois, wle, R):
    h = rois[:, R * R:].astype(np.int64)
    key = (h[:, 2] + 65536 * h[:, 3]) * 2 ** 32 + h[:, 1] * 2 ** 16 + h[:, 0]
    o = np.argsort(key, kind="stable")
    return rois[o], wle[o]


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_extract_bit_exact_against_oracle(cuda_ok, case):
    fr, para, batch = make(case)
    rois, wle, (f0, f1), dropped = run_product(fr, para, batch, start_frame=123)
    ro, wo, g0, g1 = O.extract(para, fr, batch, start_frame=123, flags=DEVICE_MODE)
    assert ro.shape[0] > 10
    assert dropped == 0
    assert rois.shape == ro.shape
    assert np.array_equal(rois, ro)
    assert (f0, f1) == (g0, g1)
    check_wle(para, rois, wle, wo)


def check_wle(para, rois, wle, wle_oracle):
    """WLE rows from extraction: equal bits to qcs_wle_estimate on the same
    records; close to the oracle's (nearest-neighbour column exact, widths
    within 1e-5 relative, molecule type equal on >= 99.5 % of records)."""
    ctx = qlib.LocContext(para, capacity=max(rois.shape[0], 1))
    own = ctx.wle(rois)
    ctx.close()
    assert np.array_equal(wle.view(np.uint32), own.view(np.uint32))
    assert np.array_equal(wle[:, 0], wle_oracle[:, 0])
    np.testing.assert_allclose(wle[:, 1:5], wle_oracle[:, 1:5], rtol=1e-5, atol=1e-6)
    assert np.mean(wle[:, 5] == wle_oracle[:, 5]) >= 0.995


@pytest.mark.parametrize("case", CASES[:2], ids=[c[0] for c in CASES[:2]])
def test_device_frames_same_as_host_frames(cuda_ok, case):
    fr, para, batch = make(case)
    a = run_product(fr, para, batch, source="normal")
    b = run_product(fr, para, batch, source="gpu")
    assert np.array_equal(a[0], b[0])
    assert np.array_equal(a[1].view(np.uint32), b[1].view(np.uint32))


@pytest.mark.skipif(not os.path.exists(O.REF_GPU_SO), reason="reference CUDA build not present")
@pytest.mark.parametrize("case", CASES[:6], ids=[c[0] for c in CASES[:6]])
def test_extract_matches_reference_cuda_build(cuda_ok, case):
    fr, para, batch = make(case)
    R = para.ROISize
    rois, wle, (f0, f1), _ = run_product(fr, para, batch, start_frame=9)
    rr, wr, g0, g1 = O.extract(para, fr, batch, start_frame=9, lib="ref_gpu")
    a_r, a_w = sort_by_key(rois, wle, R)
    b_r, b_w = sort_by_key(rr, wr, R)
    assert a_r.shape == b_r.shape
    assert np.array_equal(a_r, b_r)
    cols = slice(0, 6) if R <= 7 else slice(0, 3)
    assert np.array_equal(a_w[:, cols].view(np.uint32), b_w[:, cols].view(np.uint32))
    assert (f0, f1) == (g0, g1)


def test_full_frame_2048(cuda_ok):
    """One 2048 x 2048 camera frame (the reference's largest single-frame batch)."""
    fr, para, _ = synth.frames(1, width=2048, height=2048, density=3000, seed=31)
    para.MultiEmitterFitEn = 1
    rois, wle, _, _ = run_product(fr, para, 1)
    ro, wo, _, _ = O.extract(para, fr, 1, flags=DEVICE_MODE)
    assert ro.shape[0] > 1500
    assert np.array_equal(rois, ro)
    check_wle(para, rois, wle, wo)


def test_accumulation_reset_and_frame_range(cuda_ok):
    fr, para, batch = make(CASES[0])
    ctx = qlib.ExtractContext(para, max_batched_num=2)
    ctx.extract(fr[0:2], 10)
    n1 = ctx.accumulated()
    ctx.extract(fr[2:4], 12)
    n2 = ctx.accumulated()
    assert 0 < n1 < n2
    assert ctx.frame_range() == (10, 13)
    rois, _ = ctx.records()
    ro, _, _, _ = O.extract(para, fr, 2, start_frame=10, flags=DEVICE_MODE)
    assert np.array_equal(rois, ro)
    ctx.reset()
    assert ctx.accumulated() == 0
    assert ctx.frame_range() == (-1, -1)
    ctx.extract(fr[2:4], 50)
    rois2, _ = ctx.records()
    assert rois2.shape[0] == n2 - n1
    assert ctx.frame_range() == (50, 51)
    ctx.close()


def test_capacity_drops_and_counts(cuda_ok):
    fr, para, batch = make(CASES[0])
    ro, wo, _, _ = O.extract(para, fr, batch, flags=DEVICE_MODE)
    cap = ro.shape[0] // 3
    rois, wle, _, dropped = run_product(fr, para, batch, capacity=cap)
    assert rois.shape[0] == cap
    assert dropped == ro.shape[0] - cap
    assert np.array_equal(rois, ro[:cap])


def test_argument_errors(cuda_ok):
    fr, para, batch = make(CASES[0])
    ctx = qlib.ExtractContext(para, max_batched_num=1)
    L = qlib.load()
    a = np.ascontiguousarray(fr[:2])
    code = L.qcs_extract_molecules(ctx.h, C.c_void_p(a.ctypes.data), 2, C.byref(para), 0, 2, None)
    assert code == 3  # two frames into a one-frame context: QCS_ERR_CAPACITY
    code = L.qcs_extract_molecules(ctx.h, C.c_void_p(a.ctypes.data), 7, C.byref(para), 0, 1, None)
    assert code == 1  # unknown image source
    bad = abi.LocPara.from_buffer_copy(para)
    bad.ROISize = 9
    code = L.qcs_extract_molecules(ctx.h, C.c_void_p(a.ctypes.data), 2, C.byref(bad), 0, 1, None)
    assert code == 2
    assert ctx.accumulated() == 0
    ctx.close()


def test_pipeline_extract_then_localize_on_device(cuda_ok):
    """Records stay on the device from frames to localizations; the rows equal
    those of the host-record entry point on the same records."""
    import torch
    fr, para, batch = make(CASES[0])
    ex = qlib.ExtractContext(para, max_batched_num=batch)
    for f in range(0, fr.shape[0], batch):
        ex.extract(fr[f:f + batch], f)
    n = ex.accumulated()
    d_rois, d_wle, _ = ex.device_records()
    loc = qlib.LocContext(para)
    s = torch.cuda.Stream()
    loc.localize_device(d_rois, n, d_wle, s.cuda_stream)
    s.synchronize()
    lib = qlib.load()
    torch.cuda.synchronize()
    nv_ptr = lib.qcs_loc_device_valid_num(loc.h)
    cnt = int(torch.as_tensor(_DeviceView(nv_ptr, (1,), "<i4"), device="cuda").cpu()[0])
    rows_dev = torch.as_tensor(_DeviceView(lib.qcs_loc_device_rows(loc.h), (cnt, 12), "<f4"),
                               device="cuda").cpu().numpy()
    rois, wle = ex.records()
    rows_host, _ = loc.localize(rois, wle)
    assert cnt == rows_host.shape[0] >= n
    assert np.array_equal(rows_dev.view(np.uint32), rows_host.view(np.uint32))
    loc.close()
    ex.close()


class _DeviceView:
    def __init__(self, ptr, shape, typestr):
        self.__cuda_array_interface__ = {"shape": shape, "typestr": typestr, "data": (int(ptr), False),
                                         "version": 2}


def test_pipeline_device_count_no_host_sync(cuda_ok):
    """Frames -> extraction -> localization with the record count read on the
    device (qcs_loc_localize_device_n), several frames in a row on one stream
    with asynchronous resets: each frame's rows (qcs_loc_read_rows) equal the
    host-record entry point's rows on that frame's records."""
    import torch
    fr, para, _ = make(CASES[0])
    ex = qlib.ExtractContext(para, max_batched_num=1)
    loc = qlib.LocContext(para)
    ref = qlib.LocContext(para)
    s = torch.cuda.Stream()
    d_rois, d_wle, d_n = ex.device_records()
    for k in range(fr.shape[0]):
        ex.reset(s.cuda_stream)
        ex.extract(fr[k:k + 1], 40 + k, stream=s.cuda_stream)
        loc.localize_device_n(d_rois, d_wle, d_n, loc.capacity, s.cuda_stream)
        rows, ratios = loc.read_rows(s.cuda_stream)
        rois, wle = ex.records()
        assert rois.shape[0] > 0 and (rois[:, para.ROISize ** 2 + 2] == 40 + k).all()
        rows_h, ratios_h = ref.localize(rois, wle)
        assert np.array_equal(rows.view(np.uint32), rows_h.view(np.uint32))
        assert np.array_equal(ratios, ratios_h)
    loc.close()
    ref.close()
    ex.close()
