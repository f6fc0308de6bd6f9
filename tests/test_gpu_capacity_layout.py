"""Context buffers for any capacity: a localization context carves its cascade
state (queues, flags, the multi-emitter fits' extra rows, counters, scan
space) and the learned start points from single allocations sized by the
capacity; every part starts on a 256-byte boundary, so capacities that are not
multiples of 4 (odd ones among them) give the same rows bit for bit as a
capacity that is, through the multi-emitter cascade (2E / 3E rows moved 16
bytes at a time) and the learned path."""
import numpy as np
import pytest

from qcstorm_b200 import lib as qlib
from qcstorm_b200 import synth

pytestmark = pytest.mark.gpu


def rows_of(para, d, n, capacity, stream, net=None):
    ctx = qlib.LocContext(para, capacity=capacity)
    if net is None:
        ctx.localize_device(d.data_ptr(), n, 0, stream.cuda_stream)
    else:
        net.localize(ctx, d.data_ptr(), n, iters=2, bisections=6, stream=stream.cuda_stream)
    rows, ratios = ctx.read_rows(stream.cuda_stream)
    ctx.close()
    return rows, ratios


@pytest.mark.parametrize("gen,R,loc_type", [(synth.multi_rois, 7, 0), (synth.as3d_rois, 9, 1)])
def test_odd_capacities_give_the_same_rows(cuda_ok, gen, R, loc_type):
    import torch
    n = 1001
    rec, para, _ = gen(n, R=R, seed=77)
    para.MultiEmitterFitEn = 1
    d = torch.from_numpy(rec.view(np.int16)).cuda()
    s = torch.cuda.Stream()
    torch.cuda.synchronize()
    ref, ref_r = rows_of(para, d, n, 4096, s)
    assert ref.shape[0] > n  # second emitters appended
    for cap in (1001, 1002, 1003, 1005, 4097):
        got, got_r = rows_of(para, d, n, cap, s)
        assert got.shape == ref.shape, cap
        np.testing.assert_array_equal(got.view(np.uint32), ref.view(np.uint32))
        np.testing.assert_array_equal(got_r, ref_r)


def test_odd_capacity_learned_multi(cuda_ok):
    import torch
    n = 1001
    rec, para, _ = synth.multi_rois(n, R=7, seed=78)
    d = torch.from_numpy(rec.view(np.int16)).cuda()
    s = torch.cuda.Stream()
    torch.cuda.synchronize()
    net = qlib.LearnedNet(batch=512, seed=3, loc_type=0, roi_size=7)
    net.set_count_threshold(0.5)
    ref, _ = rows_of(para, d, n, 4096, s, net)
    for cap in (1001, 1003):
        got, _ = rows_of(para, d, n, cap, s, net)
        np.testing.assert_array_equal(got.view(np.uint32), ref.view(np.uint32))
    net.close()
