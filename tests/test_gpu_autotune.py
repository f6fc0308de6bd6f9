"""The autotuner (qcs_loc_autotune): per batch size, the fastest of one
thread per ROI and the lane-group kernel (4, 8, 16 lanes for GS2D 7x7; 8 for
the other shapes) is kept in the context, and localizations with a tuned
context give the untuned rows bit for bit (the kernels' rows are identical),
for a table forcing every lane count and for the measured one."""
import numpy as np
import pytest

from qcstorm_b200 import lib as qlib
from qcstorm_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("gen,R,lanes", [(synth.gs2d_rois, 7, (1, 4, 8, 16)), (synth.as3d_rois, 9, (1, 8)),
                                         (synth.gs2d_rois, 11, (1, 8))])
def test_autotune_table_and_identical_rows(cuda_ok, gen, R, lanes):
    import torch
    rec, para, _ = gen(6000, R=R, seed=3)
    n = rec.shape[0]
    d = torch.from_numpy(rec.view(np.int16)).cuda()
    ctx = qlib.LocContext(para, capacity=n)
    wle = torch.from_numpy(ctx.wle(rec)).cuda()
    torch.cuda.synchronize()
    s = torch.cuda.Stream()
    ctx.localize_device(d.data_ptr(), n, wle.data_ptr(), s.cuda_stream)
    base, _ = ctx.read_rows(s.cuda_stream)
    table = ctx.autotune(d.data_ptr(), wle.data_ptr(), n, stream=s.cuda_stream)
    assert table and table[-1][0] >= n
    assert all(l in lanes for _, l in table)
    for m in (300, n):
        for l in lanes + (None,):
            if l is not None:
                ctx.set_tuning([(1 << 30, l)])
            else:
                ctx.set_tuning(table)
            ctx.localize_device(d.data_ptr(), m, wle.data_ptr(), s.cuda_stream)
            got, _ = ctx.read_rows(s.cuda_stream)
            np.testing.assert_array_equal(got.view(np.uint32), base[:m].view(np.uint32))
    with pytest.raises(RuntimeError):
        ctx.set_tuning([(100, 3)])
    ctx.close()


def test_multi_emitter_stage_limits_and_identical_rows(cuda_ok, tmp_path):
    """With multi-emitter fitting the tuner also times the 2E and 3E stages with lane groups and with one
    thread per ROI; any limit gives the same rows, and the tuning survives a cache file (for this GPU and
    shape only)."""
    import torch
    rec, para, _ = synth.multi_rois(12000, R=11, seed=5)
    n = rec.shape[0]
    d = torch.from_numpy(rec.view(np.int16)).cuda()
    ctx = qlib.LocContext(para, capacity=n)
    wle = torch.from_numpy(ctx.wle(rec)).cuda()
    torch.cuda.synchronize()
    s = torch.cuda.Stream()
    ctx.localize_device(d.data_ptr(), n, wle.data_ptr(), s.cuda_stream)
    base, _ = ctx.read_rows(s.cuda_stream)
    ctx.autotune(d.data_ptr(), wle.data_ptr(), n, stream=s.cuda_stream)
    l2, l3 = ctx.tuning_multi()
    assert l2 != 0 and l3 != 0  # measured
    for limits in ((l2, l3), (-1, -1), (1 << 30, 1 << 30), (0, 0)):
        ctx.set_tuning_multi(*limits)
        ctx.localize_device(d.data_ptr(), n, wle.data_ptr(), s.cuda_stream)
        got, _ = ctx.read_rows(s.cuda_stream)
        assert got.shape == base.shape
        np.testing.assert_array_equal(got[:n].view(np.uint32), base[:n].view(np.uint32))
        np.testing.assert_array_equal(np.sort(got[n:].view(np.uint32), axis=0), np.sort(base[n:].view(np.uint32), axis=0))
    table = ctx.tuning()
    ctx.set_tuning_multi(l2, l3)
    path = tmp_path / "tuning.txt"
    ctx.save_tuning(path)
    other = qlib.LocContext(para, capacity=n)
    other.load_tuning(path)
    assert other.tuning() == table and other.tuning_multi() == (l2, l3)
    wrong = qlib.LocContext(para.copy(ROISize=7), capacity=64)
    with pytest.raises(qlib.QcsError) as e:
        wrong.load_tuning(path)
    assert e.value.code == 6  # written for another shape
    for c in (ctx, other, wrong):
        c.close()


def test_learned_iteration_cap(cuda_ok):
    """qcs_learned_autotune picks a compiled schedule whose acceptance is within 0.5 points of the best."""
    import torch
    rec, para, _ = synth.gs2d_rois(20000, R=7, seed=8)
    n = rec.shape[0]
    d = torch.from_numpy(rec.view(np.int16)).cuda()
    ctx = qlib.LocContext(para, capacity=n)
    ctx.localize_device(d.data_ptr(), n, 0, 0)
    torch.cuda.synchronize()
    feat, scale = qlib.LearnedNet.features(para, d.data_ptr(), n)
    tgt, valid = qlib.LearnedNet.targets(para, d.data_ptr(), ctx.device_rows(), scale, n)
    net = qlib.LearnedNet(batch=2048, seed=3)
    net.train(feat, tgt, valid, epochs=4, lr=2e-3)
    torch.cuda.synchronize()
    it, nb = net.autotune(ctx, d.data_ptr(), n)
    assert (it, nb) in {(2, 4), (2, 6), (2, 8), (3, 4), (3, 6), (3, 8), (4, 6), (2, 11), (3, 11), (4, 11), (5, 11),
                        (8, 11)}
    net.localize(ctx, d.data_ptr(), n, iters=it, bisections=nb)
    rows, _ = ctx.read_rows()
    assert (rows[:, 0] > 0).mean() > 0.9
    net.close()
    ctx.close()
