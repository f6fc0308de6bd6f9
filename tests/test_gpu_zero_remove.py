"""Zero-row removal on the GPU (qcs_zero_remove*), through the C ABI: equal
bits and order to the oracle (which is pinned to the reference's host build);
against the reference's CUDA build the kept rows of each frame are equal as a
set (it appends within a frame in atomic arrival order)."""
import os

import numpy as np
import pytest

import oracle_lib as O
from qcstorm_b200 import lib as qlib
from test_oracle_zero_remove_pin import localized_rows

pytestmark = pytest.mark.gpu

CASES = [(0, 0, 0), (1, 100, 139), (1, 105, 120), (1, 200, 210)]


@pytest.mark.parametrize("sort,f0,f1", CASES)
def test_zero_remove_matches_oracle(cuda_ok, sort, f0, f1):
    rows = localized_rows()
    z = qlib.ZeroRemover()
    got = z.remove(rows, sort, f0, f1)
    z.close()
    exp = O.zero_remove(rows, sort, f0, f1)
    assert got.shape == exp.shape
    assert np.array_equal(got.view(np.uint32), exp.view(np.uint32))


@pytest.mark.skipif(not os.path.exists(O.REF_GPU_SO), reason="reference CUDA build not present")
@pytest.mark.parametrize("sort,f0,f1", CASES[:3])
def test_zero_remove_matches_reference_cuda_build(cuda_ok, sort, f0, f1):
    rows = localized_rows(seed=5)
    z = qlib.ZeroRemover()
    got = z.remove(rows, sort, f0, f1)
    z.close()
    ref = O.zero_remove(rows, sort, f0, f1, "ref_gpu")
    assert got.shape == ref.shape
    if sort:
        assert np.array_equal(got[:, 11], ref[:, 11])  # same frame sequence
    key = lambda a: a[np.lexsort(a.view(np.uint32).T[::-1])]
    assert np.array_equal(key(got).view(np.uint32), key(ref).view(np.uint32))


def test_zero_remove_device_count_on_device(cuda_ok):
    """Device form with the row count read on the device (as chained after
    qcs_loc_localize_device_n): rows past the count are ignored."""
    import torch
    rows = localized_rows(seed=7)
    n = rows.shape[0]
    d_rows = torch.from_numpy(np.concatenate([rows, np.full((100, 12), 50.0, np.float32)])).cuda()
    d_out = torch.zeros((n + 100, 12), dtype=torch.float32, device="cuda")
    d_n = torch.tensor([n], dtype=torch.int32, device="cuda")
    d_k = torch.zeros(1, dtype=torch.int32, device="cuda")
    z = qlib.ZeroRemover()
    s = torch.cuda.Stream()
    z.remove_device(d_rows.data_ptr(), n + 100, d_out.data_ptr(), d_n=d_n.data_ptr(), d_nvalid=d_k.data_ptr(),
                    sort_frame=True, first_frame=100, end_frame=139, stream=s.cuda_stream)
    s.synchronize()
    k = int(d_k.cpu()[0])
    exp = O.zero_remove(rows, 1, 100, 139)
    assert k == exp.shape[0]
    assert np.array_equal(d_out.cpu().numpy()[:k].view(np.uint32), exp.view(np.uint32))
    z.close()


def test_zero_remove_capacity_and_arguments(cuda_ok):
    z = qlib.ZeroRemover(capacity=10)
    with pytest.raises(qlib.QcsError):
        z.remove(np.zeros((11, 12), np.float32))
    with pytest.raises(qlib.QcsError):
        z.remove(np.zeros((5, 12), np.float32), sort_frame=True, first_frame=9, end_frame=3)
    assert z.remove(np.zeros((0, 12), np.float32)).shape == (0, 12)
    z.close()
