"""Asynchronous host-buffer localization (qcs_loc_localize_async,
qcs_learned_localize_async, qcs_loc_finish).

The asynchronous calls enqueue the record copy, the localization and the
copy of rows and counters back without waiting; qcs_loc_finish publishes
them.  Their rows must equal the synchronous call's bit for bit (GS2D with
the WLE pre-pass on the device and with WLE rows given, multi-emitter 11x11
whose appended rows come back through the 3n row bound), also when two
contexts are used in turn on their own streams, and the learned form must
equal qcs_learned_localize_device.  A context refuses calls while one is
pending.
"""
import numpy as np
import pytest

from qcstorm_b200 import lib as qlib
from qcstorm_b200 import synth

pytestmark = pytest.mark.gpu


def pinned(a):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a).view(np.int16 if a.dtype == np.uint16 else a.dtype)).pin_memory()
    return t


def same(a, b):
    assert a.shape == b.shape
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.parametrize("case", ["gs2d", "gs2d_wle", "multi11"])
def test_async_equals_sync(cuda_ok, case):
    if case == "multi11":
        rec, para, _ = synth.multi_rois(4000, R=11, seed=3)
        para.MultiEmitterFitEn = 1
    else:
        rec, para, _ = synth.gs2d_rois(6000, seed=4)
    ctx = qlib.LocContext(para, capacity=rec.shape[0])
    wle = ctx.wle(rec) if case == "gs2d_wle" else None
    ref, ratios_ref = ctx.localize(rec, wle)
    h = pinned(rec)
    hw = pinned(wle) if wle is not None else None
    ctx.localize_async(h.data_ptr(), rec.shape[0], hw.data_ptr() if hw is not None else 0)
    got, ratios = ctx.finish()
    same(got, ref)
    np.testing.assert_array_equal(ratios, ratios_ref)
    if case == "multi11":
        assert got.shape[0] > rec.shape[0]  # appended second emitters came back
    ctx.close()


def test_two_contexts_in_turn(cuda_ok):
    import torch
    batches = [synth.gs2d_rois(5000, seed=10 + k)[0] for k in range(6)]
    para = synth.gs2d_rois(1, seed=0)[1]
    one = qlib.LocContext(para, capacity=5000)
    refs = [one.localize(b)[0] for b in batches]
    one.close()
    ctxs = [qlib.LocContext(para, capacity=5000) for _ in range(2)]
    streams = [torch.cuda.Stream() for _ in range(2)]
    hs = [pinned(b) for b in batches]
    got = [None] * len(batches)
    for k in range(len(batches)):
        c = ctxs[k % 2]
        if k >= 2:
            got[k - 2] = c.finish()[0]
        c.localize_async(hs[k].data_ptr(), 5000, stream=streams[k % 2].cuda_stream)
    for k in range(len(batches) - 2, len(batches)):
        got[k] = ctxs[k % 2].finish()[0]
    for g, r in zip(got, refs):
        same(g, r)
    for c in ctxs:
        c.close()


def test_pending_call_is_exclusive(cuda_ok):
    rec, para, _ = synth.gs2d_rois(1000, seed=5)
    ctx = qlib.LocContext(para, capacity=1000)
    h = pinned(rec)
    with pytest.raises(RuntimeError):
        ctx.finish()
    ctx.localize_async(h.data_ptr(), 1000)
    with pytest.raises(RuntimeError):
        ctx.localize(rec)
    with pytest.raises(RuntimeError):
        ctx.localize_async(h.data_ptr(), 1000)
    rows, _ = ctx.finish()
    assert rows.shape[0] == 1000
    ctx.close()


def test_learned_async_equals_device_call(cuda_ok):
    import torch
    tr, para, _ = synth.gs2d_rois(20_000, seed=21)
    ctx = qlib.LocContext(para, capacity=20_000)
    d_tr = torch.from_numpy(tr.view(np.int16)).cuda()
    ctx.localize_device(d_tr.data_ptr(), tr.shape[0])
    ctx.read_rows()
    feat, scale = qlib.LearnedNet.features(para, d_tr.data_ptr(), tr.shape[0])
    tgt, valid = qlib.LearnedNet.targets(para, d_tr.data_ptr(), ctx.device_rows(), scale, tr.shape[0])
    net = qlib.LearnedNet(batch=1024, seed=6)
    net.train(feat, tgt, valid, epochs=2, lr=2e-3)
    rec, _, _ = synth.gs2d_rois(8000, seed=22)
    d = torch.from_numpy(rec.view(np.int16)).cuda()
    s = torch.cuda.Stream()
    net.localize(ctx, d.data_ptr(), rec.shape[0], iters=2, stream=s.cuda_stream)
    ref, _ = ctx.read_rows(s.cuda_stream)
    other = qlib.LocContext(para, capacity=8000)
    h = pinned(rec)
    other.localize_async(h.data_ptr(), rec.shape[0], net=net, iters=2)
    got, _ = other.finish()
    same(got, ref)
    ctx.close()
    other.close()
    net.close()
