"""Consecutive-frame merging on the GPU (qcs_consec_*) against the
reference's own ConsecutiveFit_TypeDef built for sm_100a (oracle/_ref): the
output rows of every call (merged first rows, zeroed later rows, CRLB of the
rows that leave) and the on-time ratios equal bit for bit, over several
groups, 2D and astigmatic 3D rows, thresholds below and above one pixel.
Against the CPU oracle with the GPU's roundings the rows agree up to the
CRLB restatement's rounding (libm logf on the host) and what the next call's
merge weights carry of it; the device-resident form equals the host form."""
import numpy as np
import pytest

import oracle_lib as O
from consec_rows import consec_rows, group_sizes
from qcstorm_b200 import lib as qlib
from qcstorm_b200.abi import default_para

pytestmark = pytest.mark.gpu

CASES = [(0, 80.0, 3), (0, 250.0, 2), (1, 80.0, 4), (1, 250.0, 3)]


def product(para, rows, sizes, device=False):
    import torch
    cf = qlib.ConsecFit(capacity=int(max(sizes)))
    outs, ons = [], []
    o = 0
    for g, k in enumerate(sizes):
        chunk = rows[o:o + k]
        o += k
        end = g == len(sizes) - 1
        if device:
            d = torch.from_numpy(np.ascontiguousarray(chunk)).cuda()
            torch.cuda.synchronize()
            cf.fit_device(d.data_ptr(), k, para, is_end=end)
            outs.append(cf.read_rows())
            ons.append(cf._result()[1])
        else:
            r, on = cf.fit(chunk, para, is_end=end)
            outs.append(r)
            ons.append(on)
    cf.close()
    return outs, np.stack(ons)


@pytest.mark.parametrize("loc_type,th_nm,fpg", CASES)
def test_consec_matches_reference_cuda_build(cuda_ok, loc_type, th_nm, fpg):
    rows, counts = consec_rows(n_emitters=300, frames=12, seed=5 + loc_type, loc_type=loc_type)
    para = default_para(LocType=loc_type, ConsecFit_DistanceTh_nm=th_nm, PixelSize=100.0, QE=0.8)
    sizes = group_sizes(counts, fpg)
    ref, ref_on = O.consec(para, rows, sizes, lib="ref_gpu")
    got, got_on = product(para, rows, sizes)
    assert len(got) == len(ref)
    for a, b in zip(got, ref):
        assert a.shape == b.shape
        np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32))
    np.testing.assert_array_equal(got_on.view(np.uint32), ref_on.view(np.uint32))
    assert sum(int((b[:, 0] == 0).sum()) for b in ref) > 50


@pytest.mark.parametrize("loc_type,th_nm,fpg", CASES[:2])
def test_consec_matches_oracle(cuda_ok, loc_type, th_nm, fpg):
    rows, counts = consec_rows(n_emitters=300, frames=12, seed=9 + loc_type, loc_type=loc_type)
    para = default_para(LocType=loc_type, ConsecFit_DistanceTh_nm=th_nm, PixelSize=100.0, QE=0.8)
    sizes = group_sizes(counts, fpg)
    ora, ora_on = O.consec(para, rows, sizes, lib="oracle", gpu_rounding=1)
    got, got_on = product(para, rows, sizes)
    for a, b in zip(got, ora):
        assert a.shape == b.shape
        np.testing.assert_array_equal(np.isnan(a), np.isnan(b))
        np.testing.assert_array_equal(a[:, 11], b[:, 11])
        np.testing.assert_array_equal(a[:, 0] == 0, b[:, 0] == 0)
        # CRLB columns: CUDA logf against libm logf in a numerical second derivative
        np.testing.assert_allclose(a[:, 9:11], b[:, 9:11], rtol=5e-3, equal_nan=True)
        keep = np.r_[0:9, 11]
        np.testing.assert_allclose(a[:, keep], b[:, keep], rtol=2e-5, atol=1e-4, equal_nan=True)
    np.testing.assert_array_equal(got_on, ora_on)


def test_consec_device_form_equals_host_form(cuda_ok):
    rows, counts = consec_rows(n_emitters=300, frames=9, seed=21)
    para = default_para(LocType=0, ConsecFit_DistanceTh_nm=120.0, PixelSize=100.0, QE=0.8)
    sizes = group_sizes(counts, 3)
    a, a_on = product(para, rows, sizes)
    b, b_on = product(para, rows, sizes, device=True)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x.view(np.uint32), y.view(np.uint32))
    np.testing.assert_array_equal(a_on, b_on)


def test_consec_refuses_bad_calls(cuda_ok):
    cf = qlib.ConsecFit(capacity=10)
    para = default_para()
    with pytest.raises(RuntimeError):
        cf.fit(np.zeros((11, 12), np.float32), para)
    bad = para.copy(PixelSize=0.0)
    with pytest.raises(RuntimeError):
        cf.fit(np.zeros((2, 12), np.float32), bad)
    cf.close()
