"""Single-emitter fit with several lanes per ROI (qcs_fit_single_group_device).

The group kernel splits each loss evaluation's pixel terms and each
gradient's central-difference points over the lanes of a group, then sums in
the serial kernel's order.  Its rows must equal fit_single_kernel's
(qcs_fit_single_device) bit for bit, for every ROI size it offers, both
single-emitter kinds, every lane count and every weighted-MLE branch
(molecule types 0 / 1 / 2, WLE on and off); the WLE rows are drawn at random
so that all branches occur.
"""
import numpy as np
import pytest

from qcstorm_b200 import lib as qlib
from qcstorm_b200 import synth

pytestmark = pytest.mark.gpu


def random_wle(n, R, seed):
    rng = np.random.default_rng(seed)
    w = np.zeros((n, 6), np.float32)
    w[:, 0] = rng.uniform(1, 20, n)
    w[:, 1:5] = rng.uniform(0.6, R / 2.0, (n, 4))
    w[:, 5] = rng.integers(0, 3, n)
    return w


def rows_of(fn, loc_type, para, rec, wle, **kw):
    import torch
    n = rec.shape[0]
    d_rec = torch.from_numpy(rec.view(np.int16)).cuda()
    d_wle = torch.from_numpy(wle).cuda()
    d_loc = torch.full((n, 12), float("nan"), dtype=torch.float32, device="cuda")
    fn(loc_type, para, d_rec.data_ptr(), d_wle.data_ptr(), n, d_loc.data_ptr(), **kw)
    torch.cuda.synchronize()
    return d_loc.cpu().numpy()


CASES = [(0, 7), (0, 9), (0, 11), (0, 13), (1, 7), (1, 9), (1, 11)]


@pytest.mark.parametrize("loc_type,R", CASES)
@pytest.mark.parametrize("wle_en", [1, 0])
def test_group_fit_equals_thread_fit(cuda_ok, loc_type, R, wle_en):
    n = 3001  # ragged last block
    if loc_type == 0:
        rec, para, _ = synth.gs2d_rois(n, R=R, seed=40 + R)
    else:
        rec, para, _ = synth.as3d_rois(n, R=R, seed=50 + R)
    para.WLEEn = wle_en
    wle = random_wle(n, R, seed=R)
    ref = rows_of(qlib.fit_single_device, loc_type, para, rec, wle)
    got = rows_of(qlib.fit_single_group_device, loc_type, para, rec, wle, lanes=8)
    assert np.isfinite(ref).all()
    assert (ref[:, 0] > 0).mean() > 0.5
    np.testing.assert_array_equal(got.view(np.uint32), ref.view(np.uint32))


@pytest.mark.parametrize("lanes", [4, 16])
def test_group_fit_lane_counts(cuda_ok, lanes):
    n = 2000
    rec, para, _ = synth.gs2d_rois(n, R=7, seed=61)
    wle = random_wle(n, 7, seed=62)
    ref = rows_of(qlib.fit_single_device, 0, para, rec, wle)
    got = rows_of(qlib.fit_single_group_device, 0, para, rec, wle, lanes=lanes)
    np.testing.assert_array_equal(got.view(np.uint32), ref.view(np.uint32))


def test_group_fit_rejects_bad_lanes(cuda_ok):
    rec, para, _ = synth.as3d_rois(10, R=9, seed=1)
    with pytest.raises(RuntimeError):
        rows_of(qlib.fit_single_group_device, 1, para, rec, random_wle(10, 9, 1), lanes=4)


@pytest.mark.parametrize("loc_type,R", [(0, 5), (0, 15), (1, 13)])
def test_group_fit_refuses_compiler_rounded_sizes(cuda_ok, loc_type, R):
    """Sizes whose pixel distance is contracted as nvcc chooses: the group
    kernel could not reproduce the thread kernel's rounding, so it refuses."""
    gen = synth.gs2d_rois if loc_type == 0 else synth.as3d_rois
    rec, para, _ = gen(10, R=R, seed=2)
    with pytest.raises(RuntimeError):
        rows_of(qlib.fit_single_group_device, loc_type, para, rec, random_wle(10, R, 2), lanes=8)
