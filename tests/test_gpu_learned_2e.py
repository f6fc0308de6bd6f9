"""Learned start points of the two-emitter fits (QCS_LEARNED_GS2D_2E networks,
qcs_learned_set_two_emitter, qcs_loc_two_emitter_targets_device).

The network is the start-point MLP with 8 outputs (both emitters' positions
and peaks, the shared sigma and the background), trained on the records whose
plain two-emitter fit kept both emitters.  Its targets are checked against the
plain call's rows, its loss and gradient against the numpy restatement in
oracle/qcs_net_oracle.py, its fused start points against the numpy forward
pass.  The cascade's two-emitter stage started from them must give the
reference's rows when every fit is redone plainly (the merge of the refits into
their queue slots), and a trained pair of networks must keep the
localizations' count and accuracy against the generator's truth while most
two-emitter fits run the short schedule.
"""
import os
import sys

import numpy as np
import pytest

from qcstorm_b200 import lib as qlib
from qcstorm_b200 import synth

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import qcs_net_oracle as NO  # noqa: E402
from test_gpu_learned_counts import match_truth, plain_multi, to_dev, train_count_net  # noqa: E402

pytestmark = pytest.mark.gpu
R = 7


def two_targets(ctx, para, d, n, s):
    feat, scale = qlib.LearnedNet.features(para, d.data_ptr(), n, stream=s.cuda_stream)
    t, v = qlib.two_emitter_targets(ctx, para, d.data_ptr(), scale, n, s.cuda_stream)
    s.synchronize()
    return feat, scale, t, v


def train_two_net(para, n_train, seed, s, epochs=8):
    tr, _, _ = synth.multi_rois(n_train, R=R, seed=seed)
    d = to_dev(tr)
    ctx = qlib.LocContext(para, capacity=n_train)
    plain_multi(ctx, d, n_train, s)
    feat, _, t, v = two_targets(ctx, para, d, n_train, s)
    net2 = qlib.LearnedNet(batch=4096, seed=6, loc_type=qlib.LEARNED_GS2D_2E, roi_size=R)
    losses = net2.train(feat, t, v, epochs=epochs, lr=2e-3, stream=s.cuda_stream)
    s.synchronize()
    ctx.close()
    return net2, losses


def test_two_emitter_targets_and_gradient_match_oracle(cuda_ok):
    import torch
    rec, para, _ = synth.multi_rois(2048, R=R, seed=41)
    n = rec.shape[0]
    d = to_dev(rec)
    s = torch.cuda.Stream()
    ctx = qlib.LocContext(para, capacity=n)
    rows, _, labels = plain_multi(ctx, d, n, s)
    feat, scale, t, v = two_targets(ctx, para, d, n, s)
    t, v, sc = t.cpu().numpy(), v.cpu().numpy(), scale.cpu().numpy()
    ok = v > 0
    assert ok.sum() > 0.05 * n  # records whose two-emitter fit kept both emitters
    assert np.all(labels[ok] == 1)
    r0 = rows[:n][ok]
    c = R / 2.0
    np.testing.assert_allclose(t[ok, 0], r0[:, 1] + R // 2 - rec[ok, R * R] - c, atol=1e-5)
    np.testing.assert_allclose(t[ok, 1], r0[:, 2] + R // 2 - rec[ok, R * R + 1] - c, atol=1e-5)
    np.testing.assert_allclose(t[ok, 4], np.log(np.maximum(r0[:, 0] * para.QE, 1e-3) / sc[ok, 1]), rtol=1e-5,
                               atol=1e-5)
    np.testing.assert_allclose(t[ok, 6], r0[:, 4] - 1.3, atol=1e-6)
    np.testing.assert_allclose(t[ok, 7], (r0[:, 7] * para.QE - sc[ok, 0]) / sc[ok, 1], rtol=1e-5, atol=1e-5)
    # the second emitter of each record is one of its appended rows
    extra = rows[n:]
    for i in np.nonzero(ok)[0][:50]:
        mine = extra[extra[:, 11] == int(rec[i, R * R + 2]) + 65536 * int(rec[i, R * R + 3])]
        x1 = t[i, 2] + c - R // 2 + int(rec[i, R * R])
        assert np.min(np.abs(mine[:, 1] - x1)) < 1e-4
    assert np.all(t[~ok] == 0)
    net2 = qlib.LearnedNet(batch=n, seed=3, loc_type=qlib.LEARNED_GS2D_2E, roi_size=R)
    assert net2.n_params == NO.param_count(NO.in_width(R))
    params = net2.params()
    d_t, d_v = to_dev(t), to_dev(v)
    loss = net2.gradient(feat, d_t, d_v)
    g = net2.grads()
    loss_o, g_o, _ = NO.loss_and_grad(params, feat.cpu().numpy(), t, v)
    assert abs(loss - loss_o) <= 2e-3 * abs(loss_o)
    assert np.linalg.norm(g - g_o) <= 2e-2 * np.linalg.norm(g_o)
    net2.close()
    ctx.close()


@pytest.mark.parametrize("n", [1, 1001])
def test_two_emitter_fused_start_points(cuda_ok, n):
    import torch
    _, para, _ = synth.multi_rois(8, R=R, seed=0)
    s = torch.cuda.Stream()
    net2, _ = train_two_net(para, 8192, 43, s, epochs=2)
    rec, _, _ = synth.multi_rois(n, R=R, seed=44)
    d = to_dev(rec)
    net2.set_fused(True)
    fused = net2.start(para, d.data_ptr(), n).cpu().numpy().astype(np.float64)
    net2.fused_status()
    torch.cuda.synchronize()
    assert fused.shape == (n, 8) and np.all(np.isfinite(fused))
    feat, scale = NO.features(rec, para.Offset, para.KAdc, r=R)
    y, _ = NO.forward(net2.params(), feat)
    ref = NO.start_points_2e(y, scale[:, 0], scale[:, 1], R)
    tol = 2e-3 * max(1.0, float(np.max(np.abs(y))))
    for j in (1, 2, 4, 5, 6):
        assert np.max(np.abs(fused[:, j] - ref[:, j])) <= tol, j
    for j in (0, 3):
        assert np.max(np.abs(np.log(fused[:, j] / ref[:, j]))) <= tol, j
    assert np.max(np.abs(fused[:, 7] - ref[:, 7]) / scale[:, 1]) <= tol
    net2.close()


def test_two_emitter_stage_with_every_fit_redone_gives_plain_stage(cuda_ok):
    """With a deviance bound of ~0 every learned two-emitter fit is redone by
    the reference's fit and merged back into its slot: the call's rows equal,
    bit for bit and in order, those of the same learned call without the
    two-emitter network."""
    import torch
    rec, para, _ = synth.multi_rois(3000, R=R, seed=45)
    n = rec.shape[0]
    d = to_dev(rec)
    s = torch.cuda.Stream()
    net = qlib.LearnedNet(batch=512, seed=5, loc_type=0, roi_size=R)  # routes by the WLE classes
    net2 = qlib.LearnedNet(batch=512, seed=6, loc_type=qlib.LEARNED_GS2D_2E, roi_size=R)
    ctx = qlib.LocContext(para, capacity=n)
    net.localize(ctx, d.data_ptr(), n, iters=2, bisections=6, stream=s.cuda_stream)
    ref, ref_r = ctx.read_rows(s.cuda_stream)
    net.set_two_emitter(net2, iters=3, bisections=6, dev_th=1e-9, fallback="plain")
    net.localize(ctx, d.data_ptr(), n, iters=2, bisections=6, stream=s.cuda_stream)
    got, got_r = ctx.read_rows(s.cuda_stream)
    k2 = net.refits_2e(ctx)
    assert k2 > 0.05 * n
    assert got.shape == ref.shape
    np.testing.assert_array_equal(got.view(np.uint32), ref.view(np.uint32))
    np.testing.assert_array_equal(got_r, ref_r)
    with pytest.raises(RuntimeError):
        net.set_two_emitter(net2, iters=5, bisections=6)  # schedule not compiled
    with pytest.raises(RuntimeError):
        net2.set_two_emitter(net)  # wrong kinds
    net.set_two_emitter(None)
    ctx.close()
    net.close()
    net2.close()


def test_trained_two_emitter_starts_keep_accuracy(cuda_ok):
    """A count head and a two-emitter network trained on 100k multi-emitter
    7x7 ROIs; on 20k fresh ROIs the learned call with two-emitter start points
    (3 x 6 against the reference's 13 x 11) keeps the localizations near true
    emitters and their accuracy, with poor two-emitter fits refitted plainly
    or handed to the three-emitter fit."""
    import torch
    _, para, _ = synth.multi_rois(8, R=R, seed=0)
    s = torch.cuda.Stream()
    net, _ = train_count_net(para, 100_000, 401, s)
    net.set_count_threshold(0.5)
    net2, losses = train_two_net(para, 100_000, 402, s)
    assert losses[-1] < losses[0]
    ev, _, truth = synth.multi_rois(20_000, R=R, seed=403)
    m = ev.shape[0]
    d = to_dev(ev)
    ctx = qlib.LocContext(para, capacity=m)
    plain, _, _ = plain_multi(ctx, d, m, s)
    net.localize(ctx, d.data_ptr(), m, iters=2, bisections=6, stream=s.cuda_stream)
    one, _ = ctx.read_rows(s.cuda_stream)
    net.set_two_emitter(net2, iters=3, bisections=6, fallback="plain")
    net.localize(ctx, d.data_ptr(), m, iters=2, bisections=6, stream=s.cuda_stream)
    two_p, _ = ctx.read_rows(s.cuda_stream)
    k2 = net.refits_2e(ctx)
    net.set_two_emitter(net2, iters=3, bisections=6)  # poor fits on to the three-emitter fit
    net.localize(ctx, d.data_ptr(), m, iters=2, bisections=6, stream=s.cuda_stream)
    two, _ = ctx.read_rows(s.cuda_stream)
    assert net.refits_2e(ctx) == 0
    net.set_two_emitter(net2, iters=3, bisections=6, fallback="none")  # poor fits keep their own result
    net.localize(ctx, d.data_ptr(), m, iters=2, bisections=6, stream=s.cuda_stream)
    two_n, _ = ctx.read_rows(s.cuda_stream)
    assert net.refits_2e(ctx) == 0
    res = {}
    for name, rows in (("plain", plain), ("learned", one), ("learned_2e_refit", two_p), ("learned_2e", two),
                       ("learned_2e_none", two_n)):
        dd = match_truth(rows, ev, truth)
        ok = dd < 1.0
        res[name] = (int(ok.sum()), float(np.sqrt(np.mean(dd[ok] ** 2))), rows.shape[0])
    print("matched / rmse / rows", res, "two-emitter refits", k2)
    tp_p, rm_p, _ = res["plain"]
    for name in ("learned_2e_refit", "learned_2e", "learned_2e_none"):
        tp_2, rm_2, _ = res[name]
        assert tp_2 >= 0.97 * tp_p, name
        assert rm_2 <= 1.05 * rm_p, name
    ctx.close()
    net.close()
    net2.close()


def test_attached_two_emitter_network_outlives_owner(cuda_ok):
    # a GS2D network keeps a pointer to its attached two-emitter network:
    # destroying the attached network is refused until it is detached or its
    # owner is gone
    net = qlib.LearnedNet(batch=256, seed=1, roi_size=R)
    two = qlib.LearnedNet(batch=256, seed=2, loc_type=qlib.LEARNED_GS2D_2E, roi_size=R)
    net.set_two_emitter(two)
    with pytest.raises(qlib.QcsError) as e:
        two.close()
    assert e.value.code == 6  # QCS_ERR_STATE
    assert two.h  # still alive and usable
    net.set_two_emitter(None)
    two.close()
    assert not two.h
    two = qlib.LearnedNet(batch=256, seed=3, loc_type=qlib.LEARNED_GS2D_2E, roi_size=R)
    net.set_two_emitter(two)
    net.set_two_emitter(two)  # attaching twice counts once
    net.close()  # destroying the owner detaches
    two.close()
    assert not two.h
