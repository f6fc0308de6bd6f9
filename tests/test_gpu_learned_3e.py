"""Learned start points of the three-emitter fits (QCS_LEARNED_GS2D_3E
networks, qcs_learned_set_three_emitter, qcs_loc_set_three_emitter_capture,
qcs_loc_three_emitter_targets_device).

The network is the start-point MLP with 16 outputs (11 used: the three
emitters' positions and peaks, the shared sigma and the background), trained
on the parameters the plain three-emitter fit converged to.  Capturing them
must leave the rows unchanged; the targets are checked against the plain
call's rows (the first and second emitters in the fit's own selection order),
the loss and gradient against the numpy restatement in
oracle/qcs_net_oracle.py, the fused start points against the numpy forward
pass.  The cascade's three-emitter stage started from them must give the
reference's rows when every fit is redone plainly, and a trained network must
keep the localizations' count and accuracy against the generator's truth
while most three-emitter fits run the short schedule.
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


def three_targets(ctx, para, d, n, s):
    feat, scale = qlib.LearnedNet.features(para, d.data_ptr(), n, stream=s.cuda_stream)
    t, v = qlib.three_emitter_targets(ctx, para, d.data_ptr(), scale, n, s.cuda_stream)
    s.synchronize()
    return feat, scale, t, v


def train_three_net(para, n_train, seed, s, epochs=8):
    tr, _, _ = synth.multi_rois(n_train, R=R, seed=seed)
    d = to_dev(tr)
    ctx = qlib.LocContext(para, capacity=n_train)
    qlib.set_three_emitter_capture(ctx)
    plain_multi(ctx, d, n_train, s)
    feat, _, t, v = three_targets(ctx, para, d, n_train, s)
    net3 = qlib.LearnedNet(batch=4096, seed=7, loc_type=qlib.LEARNED_GS2D_3E, roi_size=R)
    losses = net3.train(feat, t, v, epochs=epochs, lr=2e-3, stream=s.cuda_stream)
    s.synchronize()
    ctx.close()
    return net3, losses


def test_capture_keeps_rows_and_targets_match_rows(cuda_ok):
    import torch
    rec, para, _ = synth.multi_rois(4096, R=R, seed=51)
    n = rec.shape[0]
    d = to_dev(rec)
    s = torch.cuda.Stream()
    ctx = qlib.LocContext(para, capacity=n)
    ref, ref_r, _ = plain_multi(ctx, d, n, s)
    with pytest.raises(qlib.QcsError):  # no capture yet
        three_targets(ctx, para, d, n, s)
    qlib.set_three_emitter_capture(ctx)
    rows, ratios, _ = plain_multi(ctx, d, n, s)
    np.testing.assert_array_equal(rows.view(np.uint32), ref.view(np.uint32))
    np.testing.assert_array_equal(ratios, ref_r)
    feat, scale, t, v = three_targets(ctx, para, d, n, s)
    t, v, sc = t.cpu().numpy(), v.cpu().numpy(), scale.cpu().numpy()
    ok = v > 0
    assert ok.sum() > 0.02 * n  # records whose three-emitter fit kept an emitter
    # emitter 0 of the targets is the fit's first kept emitter: the record's own row (whose x, y carry the
    # frame offset, up to ~2048 px here: float rounding up to 1.2e-4 px)
    r0 = rows[:n][ok]
    c = R / 2.0
    np.testing.assert_allclose(t[ok, 0], r0[:, 1] + R // 2 - rec[ok, R * R] - c, atol=2e-4)
    np.testing.assert_allclose(t[ok, 1], r0[:, 2] + R // 2 - rec[ok, R * R + 1] - c, atol=2e-4)
    np.testing.assert_allclose(t[ok, 6], np.log(np.maximum(r0[:, 0] * para.QE, 1e-3) / sc[ok, 1]), rtol=1e-4,
                               atol=1e-4)
    np.testing.assert_allclose(t[ok, 9], r0[:, 4] - 1.3, atol=2e-5)
    np.testing.assert_allclose(t[ok, 10], (r0[:, 7] * para.QE - sc[ok, 0]) / sc[ok, 1], rtol=1e-4, atol=1e-4)
    # emitter 1 is the second kept emitter where the fit kept two: one of the record's appended rows
    extra = rows[n:]
    frames = rec[:, R * R + 2].astype(np.int64) + 65536 * rec[:, R * R + 3].astype(np.int64)
    checked = 0
    for i in np.nonzero(ok)[0]:
        mine = extra[extra[:, 11] == frames[i]]
        if mine.shape[0] == 0:
            continue
        x1 = t[i, 2] + c - R // 2 + int(rec[i, R * R])
        if np.min(np.abs(mine[:, 1] - x1)) < 2e-4:
            checked += 1
    assert checked > 0
    assert np.all(t[~ok] == 0)
    # loss and gradient of a three-emitter network (16 outputs) against the numpy restatement
    net3 = qlib.LearnedNet(batch=n, seed=3, loc_type=qlib.LEARNED_GS2D_3E, roi_size=R)
    assert net3.n_params == NO.param_count(NO.in_width(R), 16)
    params = net3.params()
    y = net3.forward(feat).cpu().numpy()
    assert y.shape == (n, 16)
    d_t, d_v = to_dev(t), to_dev(v)
    loss = net3.gradient(feat, d_t, d_v)
    g = net3.grads()
    loss_o, g_o, y_o = NO.loss_and_grad(params, feat.cpu().numpy(), t, v, n_out=16)
    assert np.max(np.abs(y - y_o)) <= 2e-3 * max(1.0, np.max(np.abs(y_o)))
    assert abs(loss - loss_o) <= 2e-3 * abs(loss_o)
    assert np.linalg.norm(g - g_o) <= 2e-2 * np.linalg.norm(g_o)
    net3.close()
    ctx.close()


@pytest.mark.parametrize("n", [1, 1001])
def test_three_emitter_fused_start_points(cuda_ok, n):
    import torch
    _, para, _ = synth.multi_rois(8, R=R, seed=0)
    s = torch.cuda.Stream()
    net3, _ = train_three_net(para, 8192, 53, s, epochs=2)
    rec, _, _ = synth.multi_rois(n, R=R, seed=54)
    d = to_dev(rec)
    net3.set_fused(True)
    fused = net3.start(para, d.data_ptr(), n).cpu().numpy().astype(np.float64)
    net3.fused_status()
    net3.set_fused(False)
    layered = net3.start(para, d.data_ptr(), n).cpu().numpy().astype(np.float64)
    torch.cuda.synchronize()
    assert fused.shape == (n, 11) and np.all(np.isfinite(fused))
    feat, scale = NO.features(rec, para.Offset, para.KAdc, r=R)
    y, _ = NO.forward(net3.params(), feat, n_out=16)
    ref = NO.start_points_3e(y, scale[:, 0], scale[:, 1], R)
    tol = 2e-3 * max(1.0, float(np.max(np.abs(y))))
    for got in (fused, layered):
        for j in (1, 2, 4, 5, 7, 8, 9):
            assert np.max(np.abs(got[:, j] - ref[:, j])) <= tol, j
        for j in (0, 3, 6):
            assert np.max(np.abs(np.log(got[:, j] / ref[:, j]))) <= tol, j
        assert np.max(np.abs(got[:, 10] - ref[:, 10]) / scale[:, 1]) <= tol
    net3.close()


@pytest.mark.parametrize("r", [R, 11])
def test_three_emitter_stage_with_every_fit_redone_gives_plain_stage(cuda_ok, r):
    """With a deviance bound of ~0 every learned three-emitter fit is redone by
    the reference's fit and merged back into its slot: the call's rows equal,
    bit for bit and in order, those of the same learned call without the
    three-emitter network (7x7 and 11x11, the three-emitter queue short
    enough for the warp-per-ROI kernel).  The plain 11x11 cascade sends
    almost no record to the three-emitter fit (~18 per 100,000), so at 11x11
    the learned count classes route every record there (a class threshold of
    0.01 on an untrained network)."""
    import torch
    rec, para, _ = synth.multi_rois(3000, R=r, seed=55)
    n = rec.shape[0]
    d = to_dev(rec)
    s = torch.cuda.Stream()
    net = qlib.LearnedNet(batch=512, seed=5, loc_type=0, roi_size=r)  # 7x7: routes by the WLE classes
    if r == 11:
        net.set_count_threshold(0.01)
    net3 = qlib.LearnedNet(batch=512, seed=6, loc_type=qlib.LEARNED_GS2D_3E, roi_size=r)
    ctx = qlib.LocContext(para, capacity=n)
    net.localize(ctx, d.data_ptr(), n, iters=2, bisections=6, stream=s.cuda_stream)
    ref, ref_r = ctx.read_rows(s.cuda_stream)
    net.set_three_emitter(net3, iters=4, bisections=6, dev_th=1e-9)
    net.localize(ctx, d.data_ptr(), n, iters=2, bisections=6, stream=s.cuda_stream)
    got, got_r = ctx.read_rows(s.cuda_stream)
    k3 = net.refits_3e(ctx)
    assert k3 > (0.02 if r == 7 else 0.5) * n  # every fit of the three-emitter stage redone
    assert got.shape == ref.shape
    np.testing.assert_array_equal(got.view(np.uint32), ref.view(np.uint32))
    np.testing.assert_array_equal(got_r, ref_r)
    with pytest.raises(RuntimeError):
        net.set_three_emitter(net3, iters=5, bisections=6)  # schedule not compiled
    with pytest.raises(RuntimeError):
        net3.set_three_emitter(net)  # wrong kinds
    net.set_three_emitter(None)
    ctx.close()
    net.close()
    net3.close()


def test_trained_three_emitter_starts_keep_accuracy(cuda_ok):
    """A count head and a three-emitter network trained on 100k multi-emitter
    7x7 ROIs; on 20k fresh ROIs the learned call with three-emitter start
    points (4 x 6 against the reference's 16 x 11, poor fits refitted plainly)
    keeps the localizations near true emitters and their accuracy."""
    import torch
    _, para, _ = synth.multi_rois(8, R=R, seed=0)
    s = torch.cuda.Stream()
    net, _ = train_count_net(para, 100_000, 501, s)
    net.set_count_threshold(0.5)
    net3, losses = train_three_net(para, 100_000, 502, s)
    assert losses[-1] < losses[0]
    ev, _, truth = synth.multi_rois(20_000, R=R, seed=503)
    m = ev.shape[0]
    d = to_dev(ev)
    ctx = qlib.LocContext(para, capacity=m)
    plain, _, _ = plain_multi(ctx, d, m, s)
    net.localize(ctx, d.data_ptr(), m, iters=2, bisections=6, stream=s.cuda_stream)
    one, _ = ctx.read_rows(s.cuda_stream)
    net.set_three_emitter(net3, iters=4, bisections=6)
    net.localize(ctx, d.data_ptr(), m, iters=2, bisections=6, stream=s.cuda_stream)
    three, _ = ctx.read_rows(s.cuda_stream)
    k3 = net.refits_3e(ctx)
    net.set_three_emitter(net3, iters=4, bisections=6, dev_th=-1.0)  # no plain refits
    net.localize(ctx, d.data_ptr(), m, iters=2, bisections=6, stream=s.cuda_stream)
    three_nr, _ = ctx.read_rows(s.cuda_stream)
    assert net.refits_3e(ctx) == 0
    res = {}
    for name, rows in (("plain", plain), ("learned", one), ("learned_3e", three), ("learned_3e_no_refit", three_nr)):
        dd = match_truth(rows, ev, truth)
        ok = dd < 1.0
        res[name] = (int(ok.sum()), float(np.sqrt(np.mean(dd[ok] ** 2))), rows.shape[0])
    print("matched / rmse / rows", res, "three-emitter refits", k3)
    tp_p, rm_p, _ = res["plain"]
    for name in ("learned_3e", "learned_3e_no_refit"):
        tp_3, rm_3, _ = res[name]
        assert tp_3 >= 0.97 * tp_p, name
        assert rm_3 <= 1.05 * rm_p, name
    ctx.close()
    net.close()
    net3.close()


def test_attached_three_emitter_network_outlives_owner(cuda_ok):
    net = qlib.LearnedNet(batch=256, seed=1, roi_size=R)
    three = qlib.LearnedNet(batch=256, seed=2, loc_type=qlib.LEARNED_GS2D_3E, roi_size=R)
    net.set_three_emitter(three)
    with pytest.raises(qlib.QcsError) as e:
        three.close()
    assert e.value.code == 6  # QCS_ERR_STATE
    net.set_three_emitter(None)
    three.close()
    assert not three.h
    with pytest.raises(RuntimeError):  # three-emitter networks are MLPs
        qlib.LearnedNet(batch=256, seed=2, loc_type=qlib.LEARNED_GS2D_3E, roi_size=R, arch="conv")
    net.close()
