"""Learned emitter-count classes and the learned multi-emitter localization
(qcs_learned_*counts*, qcs_loc_count_labels_device, qcs_fit_from_start_classes_device,
qcs_learned_localize_device / _n with multi-emitter fitting on).

The count head's loss, gradient and classes are checked against the numpy
restatement in oracle/qcs_net_oracle.py.  The learned multi-emitter call is
the reference's cascade (bfgs_top.cu:26-204) with its single-emitter stage
started from given points: when every fit is refitted plainly its rows equal
the plain call's bit for bit, and when the classes are the plain cascade's own
outcome (each record sent straight to the stage that plain fitting reaches)
the call gives the plain call's rows as a set, in another order of the
appended second emitters.  A network trained on ROIs labelled by the plain
cascade then routes fresh ROIs: it must agree with the plain outcome on most
ROIs and keep the localizations' count and accuracy against the generator's
truth.
"""
import os
import sys

import numpy as np
import pytest

from qcstorm_b200 import lib as qlib
from qcstorm_b200 import synth

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import qcs_net_oracle as NO  # noqa: E402

pytestmark = pytest.mark.gpu
R = 7


def to_dev(a):
    import torch
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint16:
        a = a.view(np.int16)
    return torch.from_numpy(a).cuda()


def naive_start(rec, para):
    """The plain fit's own pre-estimate (centre, edge-mean background, sigma 1.3)."""
    e = np.maximum((rec[:, :49].astype(np.float32) - para.Offset) * para.KAdc, 1.0).reshape(-1, 7, 7)
    m1 = np.minimum(e[:, 0, :].mean(1) * 7, e[:, 6, :].mean(1) * 7)
    m3 = np.minimum(e[:, :, 0].mean(1) * 7, e[:, :, 6].mean(1) * 7)
    bkg = (m1 + m3) / 2 / 7
    peak = np.maximum(e[:, 3, 3] - bkg, 1.0)
    st = np.stack([peak, np.full_like(peak, 3.5), np.full_like(peak, 3.5), np.full_like(peak, 1.3), bkg], 1)
    return np.ascontiguousarray(st, np.float32)


def plain_multi(ctx, d, n, s):
    import torch
    ctx.localize_device(d.data_ptr(), n, 0, s.cuda_stream)
    rows, ratios = ctx.read_rows(s.cuda_stream)
    labels = qlib.count_labels(ctx, n, s.cuda_stream)
    s.synchronize()  # the library's streams are not ordered with torch's
    return rows, ratios, labels.cpu().numpy()


def classes_host(net, para, d, n, s=None):
    import torch
    _, cls = net.classes(para, d.data_ptr(), n, stream=s.cuda_stream if s is not None else 0)
    torch.cuda.synchronize()
    return cls.cpu().numpy()


def sorted_rows(rows):
    u = np.ascontiguousarray(rows, np.float32).view(np.uint32)
    return u[np.lexsort(u.T[::-1])]


def test_count_loss_gradient_and_classes_match_oracle(cuda_ok):
    rec, para, _ = synth.multi_rois(512, R=R, seed=12)
    d = to_dev(rec)
    n = rec.shape[0]
    feat, scale = qlib.LearnedNet.features(para, d.data_ptr(), n)
    ctx = qlib.LocContext(para, capacity=n)
    import torch
    s = torch.cuda.Stream()
    rows, _, labels = plain_multi(ctx, d, n, s)
    d_rows = to_dev(rows[:n].astype(np.float32))  # kept alive while the kernel reads it
    t, v = qlib.LearnedNet.targets(para, d.data_ptr(), d_rows.data_ptr(), scale, n)
    cls = np.random.default_rng(0).integers(-1, 3, n).astype(np.float32)
    d_cls = to_dev(cls)
    net = qlib.LearnedNet(batch=512, seed=3)
    net.train(feat, t, v, epochs=40, lr=5e-3, classes=to_dev(labels.astype(np.float32)))
    params = net.params()
    loss = net.gradient(feat, t, v, classes=d_cls)
    g = net.grads()
    loss_o, g_o, y_o = NO.loss_and_grad(params, feat.cpu().numpy(), t.cpu().numpy(), v.cpu().numpy(), cls)
    assert abs(loss - loss_o) <= 2e-3 * abs(loss_o)
    o = 0
    for size in (64 * 128, 128, 128 * 128, 128, 128 * 8, 8):
        a, b = g[o:o + size], g_o[o:o + size]
        o += size
        assert np.linalg.norm(a - b) <= 2e-2 * np.linalg.norm(b) + 1e-7, (size, np.linalg.norm(a - b), np.linalg.norm(b))
    # classes of the fused kernel and of the layer-by-layer path against the oracle's rule
    lg = y_o[:, NO.COUNT0:NO.COUNT0 + NO.CLASSES]
    p = np.exp(lg - lg.max(1, keepdims=True))
    p /= p.sum(1, keepdims=True)
    assert len(np.unique(NO.count_class(lg, 0.5))) >= 2  # the trained head does not answer one class for all
    for th in (0.5, 0.8):
        net.set_count_threshold(th)
        ref = NO.count_class(lg, th)
        near = (np.abs(p[:, 2] - th) < 0.02) | (np.abs(p[:, 1] + p[:, 2] - th) < 0.02)
        for fused in (True, False):
            net.set_fused(fused)
            c = classes_host(net, para, d, n)
            assert set(np.unique(c)) <= {0, 1, 2}
            assert np.all((c == ref) | near)
        net.set_fused(True)
        net.fused_status()
    net.set_count_threshold(0.0)
    assert net.count_threshold() == 0.0
    with pytest.raises(RuntimeError):
        net.set_count_threshold(1.5)
    ctx.close()
    net.close()


def test_count_labels_follow_the_cascade(cuda_ok):
    """Labels of a plain multi-emitter call: as many records with a label >= 1
    as the 2E queue held, as many with label 2 as the 3E queue held."""
    import torch
    rec, para, _ = synth.multi_rois(20_000, R=R, seed=21)
    n = rec.shape[0]
    d = to_dev(rec)
    ctx = qlib.LocContext(para, capacity=n)
    s = torch.cuda.Stream()
    _, ratios, labels = plain_multi(ctx, d, n, s)
    assert set(np.unique(labels)) <= {0.0, 1.0, 2.0}
    assert int((labels >= 1).sum()) == int(round(ratios[1] * n))
    assert int((labels == 2).sum()) == int(round(ratios[2] * n))
    assert (labels == 1).sum() > 0 and (labels == 2).sum() > 0
    ctx.close()


def test_learned_multi_with_refits_reproduces_plain_cascade(cuda_ok):
    """A deviance bound no fit meets: every single-queue record is refitted
    plainly, and the refit decides which rejects go on to the 2E fit, so the
    rows (second emitters and CRLB included) equal the plain call's bit for
    bit; with all-zero classes passed too."""
    import torch
    rec, para, _ = synth.multi_rois(20_000, R=R, seed=31)
    n = rec.shape[0]
    d = to_dev(rec)
    ctx = qlib.LocContext(para, capacity=n)
    s = torch.cuda.Stream()
    plain, ratios, _ = plain_multi(ctx, d, n, s)
    st = to_dev(naive_start(rec, para))
    zeros = torch.zeros(n, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    for d_cls in (0, zeros.data_ptr()):
        qlib.fit_from_start(ctx, d.data_ptr(), n, st.data_ptr(), iters=2, dev_th=1e-6, stream=s.cuda_stream,
                            d_classes=d_cls)
        got, r2 = ctx.read_rows(s.cuda_stream)
        assert got.shape == plain.shape
        np.testing.assert_array_equal(got.view(np.uint32), plain.view(np.uint32))
        np.testing.assert_array_equal(np.asarray(r2), np.asarray(ratios))
        assert ctx_refits(ctx) == int(round(ratios[0] * n))  # the whole single-emitter queue
    ctx.close()


def ctx_refits(ctx):
    import ctypes as C
    k = C.c_int(0)
    qlib.check(qlib.load().qcs_learned_refit_num(ctx.h, C.byref(k)))
    return k.value


def test_classes_from_the_plain_outcome_give_the_plain_rows(cuda_ok):
    """Classes equal to the plain cascade's outcome send each multi-emitter
    record straight to the stage that plain fitting reaches; with every
    single fit refitted plainly, the rows are the plain call's rows (as a
    set: the second emitters are appended in another order)."""
    import torch
    rec, para, _ = synth.multi_rois(20_000, R=R, seed=41)
    n = rec.shape[0]
    d = to_dev(rec)
    ctx = qlib.LocContext(para, capacity=n)
    s = torch.cuda.Stream()
    plain, ratios, labels = plain_multi(ctx, d, n, s)
    st = to_dev(naive_start(rec, para))
    d_cls = to_dev(labels.astype(np.uint8))
    qlib.fit_from_start(ctx, d.data_ptr(), n, st.data_ptr(), iters=2, dev_th=1e-6, stream=s.cuda_stream,
                        d_classes=d_cls.data_ptr())
    got, r2 = ctx.read_rows(s.cuda_stream)
    assert got.shape == plain.shape
    np.testing.assert_array_equal(got[:n].view(np.uint32), plain[:n].view(np.uint32))
    np.testing.assert_array_equal(sorted_rows(got), sorted_rows(plain))
    # only the records the plain cascade kept single are fitted (and here refitted) single
    assert ctx_refits(ctx) == int((labels == 0).sum())
    assert int(round(r2[0] * n)) == int((labels == 0).sum()) < int(round(ratios[0] * n))
    ctx.close()


def match_truth(rows, rec, truth, first_frame=1):
    """Each row's distance (px) to the nearest true emitter of its record
    (record = frame - first_frame), in ROI coordinates."""
    ok = rows[:, 0] > 0
    rows = rows[ok]
    rid = rows[:, 11].astype(np.int64) - first_frame
    hx = rec[rid, R * R].astype(np.float64)
    hy = rec[rid, R * R + 1].astype(np.float64)
    fx = rows[:, 1] - hx + R // 2
    fy = rows[:, 2] - hy + R // 2
    dx = truth["x"][rid] - fx[:, None]
    dy = truth["y"][rid] - fy[:, None]
    dist = np.sqrt(np.nanmin(dx * dx + dy * dy, axis=1))
    return dist


def train_count_net(para, n_train, seed, stream):
    """Network trained on multi-emitter ROIs labelled by the plain cascade:
    start-point targets from the records it kept single, classes from its
    outcome."""
    import torch
    tr, _, _ = synth.multi_rois(n_train, R=R, seed=seed)
    d_tr = to_dev(tr)
    ctx = qlib.LocContext(para, capacity=n_train)
    rows, _, labels = plain_multi(ctx, d_tr, n_train, stream)
    sh = stream.cuda_stream
    feat, scale = qlib.LearnedNet.features(para, d_tr.data_ptr(), n_train, stream=sh)
    tgt, valid = qlib.LearnedNet.targets(para, d_tr.data_ptr(), ctx.device_rows(), scale, n_train, stream=sh)
    stream.synchronize()
    d_lab = to_dev(labels.astype(np.float32))
    valid = valid * (d_lab == 0).float()
    torch.cuda.synchronize()
    net = qlib.LearnedNet(batch=4096, seed=5)
    losses = net.train(feat, tgt, valid, epochs=8, lr=2e-3, stream=sh, classes=d_lab)
    torch.cuda.synchronize()
    ctx.close()
    return net, losses


def test_trained_count_head_routes_multi_emitter_rois(cuda_ok):
    """Train on 150k multi-emitter 7x7 ROIs (1-3 emitters, pairwise 1-3 px);
    on 30k fresh ROIs the classes agree with the plain cascade's outcome on
    most ROIs, and the routed learned call keeps the number of
    localizations near truth emitters and their accuracy."""
    import torch
    _, para, _ = synth.multi_rois(10, R=R, seed=0)
    s = torch.cuda.Stream()
    net, losses = train_count_net(para, 150_000, 301, s)
    assert losses[-1] < losses[0]
    ev, _, truth = synth.multi_rois(30_000, R=R, seed=302)
    m = ev.shape[0]
    d_ev = to_dev(ev)
    ctx = qlib.LocContext(para, capacity=m)
    plain, ratios, labels = plain_multi(ctx, d_ev, m, s)
    net.set_count_threshold(0.5)
    cls = classes_host(net, para, d_ev, m, s)
    agree = float((cls == labels).mean())
    conf = np.zeros((3, 3), int)
    np.add.at(conf, (labels.astype(int), cls.astype(int)), 1)
    net.localize(ctx, d_ev.data_ptr(), m, iters=2, bisections=6, stream=s.cuda_stream)
    learned, r_l = ctx.read_rows(s.cuda_stream)
    dp, dl = match_truth(plain, ev, truth), match_truth(learned, ev, truth)
    tp_p, tp_l = int((dp < 1.0).sum()), int((dl < 1.0).sum())
    rm_p = float(np.sqrt(np.mean(dp[dp < 1.0] ** 2)))
    rm_l = float(np.sqrt(np.mean(dl[dl < 1.0] ** 2)))
    print("agree %.3f confusion (rows plain 0/1/2, cols learned) %s; rows plain %d learned %d; matched %d / %d; "
          "rmse %.4f / %.4f; single-stage fits %.0f / %.0f" % (
              agree, conf.tolist(), plain.shape[0], learned.shape[0], tp_p, tp_l, rm_p, rm_l, ratios[0] * m,
              r_l[0] * m))
    assert agree >= 0.80
    assert conf[1:, 1:].sum() >= 0.6 * conf[1:, :].sum()  # most multi-stage ROIs are routed
    assert tp_l >= 0.97 * tp_p
    assert rm_l <= 1.05 * rm_p
    assert r_l[0] < ratios[0]  # fewer single-emitter fits
    ctx.close()
    net.close()


def test_device_count_learned_localization(cuda_ok):
    """qcs_learned_localize_device_n with the count in device memory equals the
    host-count call on the same records."""
    import torch
    _, para, _ = synth.multi_rois(10, R=R, seed=0)
    s = torch.cuda.Stream()
    net, _ = train_count_net(para, 40_000, 401, s)
    net.set_count_threshold(0.6)
    ev, _, _ = synth.multi_rois(12_000, R=R, seed=402)
    m = ev.shape[0]
    # the buffer holds max_n records, as an extraction buffer does
    d_ev = to_dev(np.concatenate([ev, np.zeros((16_000 - m, ev.shape[1]), np.uint16)]))
    ctx = qlib.LocContext(para, capacity=16_000)
    d_wle = torch.empty((m, 6), dtype=torch.float32, device="cuda")
    wle = ctx.wle(ev)
    d_wle.copy_(torch.from_numpy(wle))
    torch.cuda.synchronize()
    net.localize(ctx, d_ev.data_ptr(), m, d_wle=d_wle.data_ptr(), iters=2, bisections=6, stream=s.cuda_stream)
    a, _ = ctx.read_rows(s.cuda_stream)
    d_n = torch.tensor([m], dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    net.localize_n(ctx, d_ev.data_ptr(), d_wle.data_ptr(), d_n.data_ptr(), 16_000, iters=2, bisections=6,
                   stream=s.cuda_stream)
    b, _ = ctx.read_rows(s.cuda_stream)
    np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32))
    net.fused_status()
    ctx.close()
    net.close()
