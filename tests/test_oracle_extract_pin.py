"""ROI extraction oracle pinned against the reference's own ExtractMolecules.

The reference (SubregionExtraction/LDROIExtraction*.cu) is built for the host
(oracle/build_ref.py) and run on seeded synthetic frames; the oracle with
flags 0 (separately rounded taps, variance summed in pixel order, the order
that one-block-at-a-time run adds in) must give the same records, WLE rows and
frame range, bit for bit and in the same order.  The device arithmetic
(fused-multiply-add taps, exact-sum variance) is a separate oracle mode; it
is checked here to agree with the host mode on the same cases, which it does
unless a threshold falls between the two variances.
"""
import numpy as np
import pytest

import oracle_lib as O
from qcstorm_b200 import synth

pytestmark = pytest.mark.skipif(O.ref_host() is None, reason="reference host build not present")

# (name, width, height, frames, batch, LocType, MultiEmitterFitEn, ROISize, density, seed)
CASES = [
    ("gs2d_multi_r7", 128, 96, 3, 2, 0, 1, 7, 40, 11),
    ("gs2d_single_r7", 128, 96, 3, 2, 0, 0, 7, 40, 12),
    ("as3d_r9_odd_width", 100, 80, 2, 1, 1, 0, 9, 30, 13),
    ("as3d_multi_r11", 144, 120, 2, 2, 1, 1, 11, 30, 14),
    ("gs2d_multi_r11_batch4", 160, 128, 4, 4, 0, 1, 11, 40, 15),
    ("gs2d_single_r5_small", 48, 40, 3, 3, 0, 0, 5, 8, 16),
    ("gs2d_multi_r13_ragged", 97, 83, 3, 2, 0, 1, 13, 25, 17),
    ("gs2d_single_r17", 128, 128, 1, 1, 0, 0, 17, 20, 18),
    ("dense_gs2d_multi_r7", 128, 128, 2, 2, 0, 1, 7, 200, 19),
]


def make(case):
    name, W, H, nf, batch, lt, multi, R, dens, seed = case
    fr, para, _ = synth.frames(nf, width=W, height=H, density=dens, seed=seed)
    para.LocType, para.MultiEmitterFitEn, para.ROISize = lt, multi, R
    return fr, para, batch


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_extract_bit_exact_against_reference_host_build(case):
    fr, para, batch = make(case)
    ro, wo, f0o, f1o = O.extract(para, fr, batch, start_frame=70000, flags=0, lib="oracle")
    rr, wr, f0r, f1r = O.extract(para, fr, batch, start_frame=70000, flags=0, lib="ref")
    assert ro.shape[0] > 0
    assert ro.shape == rr.shape
    assert np.array_equal(ro, rr)
    assert np.array_equal(wo.view(np.uint32), wr.view(np.uint32))
    assert (f0o, f1o) == (f0r, f1r) == (70000, 70000 + fr.shape[0] - 1)


@pytest.mark.parametrize("case", CASES[:5], ids=[c[0] for c in CASES[:5]])
def test_device_arithmetic_mode_agrees_with_host_mode(case):
    fr, para, batch = make(case)
    a = O.extract(para, fr, batch, flags=0)
    b = O.extract(para, fr, batch, flags=O.EXTRACT_FMA_CONV | O.EXTRACT_EXACT_VARIANCE)
    assert np.array_equal(a[0], b[0])
    assert np.array_equal(a[1].view(np.uint32), b[1].view(np.uint32))


def test_header_words_and_frame_split():
    """Header [x, y, frame % 65536, frame / 65536, type] with frames past 65535."""
    fr, para, batch = make(CASES[0])
    rois, _, _, _ = O.extract(para, fr, batch, start_frame=65535)
    R = para.ROISize
    h = rois[:, R * R:].astype(np.int64)
    frame = h[:, 2] + 65536 * h[:, 3]
    assert set(np.unique(frame)) <= {65535, 65536, 65537}
    assert (h[:, 0] >= R // 2).all() and (h[:, 0] < para.ImageWidth - R // 2).all()
    assert (h[:, 1] >= R // 2).all() and (h[:, 1] < para.ImageHigh - R // 2).all()
    # pixel order within a batch: (frame, y, x) ascending
    key = frame * 2 ** 32 + h[:, 1] * 2 ** 16 + h[:, 0]
    assert (np.diff(key) > 0).all()
    # the cut is the raw frame around the centre
    i = 0
    f, y, x = int(frame[i] - 65535), int(h[i, 1]), int(h[i, 0])
    ref = fr[f, y - R // 2:y + R // 2 + 1, x - R // 2:x + R // 2 + 1]
    assert np.array_equal(rois[i, :R * R].reshape(R, R), ref)


def test_empty_frames_give_no_records():
    fr = np.full((2, 64, 64), 100, np.uint16)
    _, para, _ = synth.frames(1, width=64, height=64, density=0, seed=1)
    rois, wle, f0, f1 = O.extract(para, fr, 2, start_frame=5)
    assert rois.shape[0] == 0 and wle.shape[0] == 0
    assert (f0, f1) == (5, 6)
    rr, _, _, _ = O.extract(para, fr, 2, start_frame=5, lib="ref")
    assert rr.shape[0] == 0
