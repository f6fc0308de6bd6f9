"""Learned start points for the other single-emitter shapes: GS2D 9x9 and
11x11, AS3D 7x7, 9x9 and 11x11 (qcs_learned_create_for and the same entry
points as the GS2D 7x7 network).

Features, targets, forward pass and gradient against the numpy restatement
in oracle/qcs_net_oracle.py; the fused tcgen05 inference (128 input features,
records bulk-copied in tiles whose ragged end is not a whole number of
16-byte blocks) against the layer-by-layer path and the numpy forward pass;
then networks trained on the GPU: fits from their start points with a short
schedule reach the plain fits' position (and, for AS3D, z) RMSE against the
generator's truth.
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

SHAPES = [(0, 9), (0, 11), (1, 7), (1, 9), (1, 11)]


def gen(loc_type, R, n, seed):
    return synth.as3d_rois(n, R=R, seed=seed) if loc_type == 1 else synth.gs2d_rois(n, R=R, seed=seed)


def to_dev(a):
    import torch
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint16:
        a = a.view(np.int16)
    return torch.from_numpy(a).cuda()


def plain_rows(rec, para):
    ctx = qlib.LocContext(para, capacity=rec.shape[0])
    rows, _ = ctx.localize(rec)
    ctx.close()
    return rows


def start_from_y(y, scale, R, loc_type):
    """The start transform of the network outputs (qcs_learned.cu start_from_outputs)."""
    lo, rng = scale[:, 0].astype(np.float64), scale[:, 1].astype(np.float64)
    win, smax = (2.5, 4.0) if loc_type == 1 else (1.5, 3.0)
    cols = [rng * np.exp(np.clip(y[:, 3], -6, 3)), R / 2.0 + np.clip(y[:, 0], -win, win),
            R / 2.0 + np.clip(y[:, 1], -win, win), np.clip(NO.SIGMA0 + y[:, 2], 0.6, smax)]
    if loc_type == 1:
        cols.append(np.clip(NO.SIGMA0 + y[:, 5], 0.6, smax))
    cols.append(np.maximum(lo + rng * y[:, 4], 1.0))
    return np.stack(cols, 1)


def assert_start_close(a, b, scale, tol):
    """Start points agree to `tol` in network-output units."""
    rng = scale[:, 1].astype(np.float64)
    assert np.max(np.abs(np.log(a[:, 0] / b[:, 0]))) <= tol
    assert np.max(np.abs(a[:, 1:-1] - b[:, 1:-1])) <= tol
    assert np.max(np.abs(a[:, -1] - b[:, -1]) / rng) <= tol


@pytest.mark.parametrize("loc_type,R", SHAPES)
def test_shape_features_targets_gradient_match_oracle(cuda_ok, loc_type, R):
    rec, para, _ = gen(loc_type, R, 512, 11 + R)
    d = to_dev(rec)
    n = rec.shape[0]
    feat, scale = qlib.LearnedNet.features(para, d.data_ptr(), n)
    f_o, s_o = NO.features(rec, para.Offset, para.KAdc, r=R)
    assert feat.shape[1] == NO.in_width(R)
    np.testing.assert_allclose(feat.cpu().numpy(), f_o, rtol=2e-6, atol=2e-6)
    np.testing.assert_array_equal(scale.cpu().numpy(), s_o)
    rows = plain_rows(rec, para)
    d_rows = to_dev(rows.astype(np.float32))  # kept alive while the kernel reads it
    t, v = qlib.LearnedNet.targets(para, d.data_ptr(), d_rows.data_ptr(), scale, n)
    t_o, v_o = NO.targets(rec, rows, s_o, para.QE, r=R, loc_type=loc_type)
    np.testing.assert_array_equal(v.cpu().numpy(), v_o)
    np.testing.assert_allclose(t.cpu().numpy(), t_o, rtol=1e-5, atol=1e-5)
    net = qlib.LearnedNet(batch=512, seed=3, loc_type=loc_type, roi_size=R)
    assert net.n_params == NO.param_count(NO.in_width(R))
    params = net.params()
    loss = net.gradient(feat, t, v)
    g = net.grads()
    loss_o, g_o, _ = NO.loss_and_grad(params, feat.cpu().numpy(), t.cpu().numpy(), v.cpu().numpy())
    assert abs(loss - loss_o) <= 2e-3 * abs(loss_o)
    o = 0
    for size in (NO.in_width(R) * 128, 128, 128 * 128, 128, 128 * 8, 8):
        a, b = g[o:o + size], g_o[o:o + size]
        o += size
        assert np.linalg.norm(a - b) <= 2e-2 * np.linalg.norm(b) + 1e-7, (size, np.linalg.norm(a - b))
    net.close()


@pytest.mark.parametrize("loc_type,R", SHAPES)
@pytest.mark.parametrize("n", [1, 1001])
def test_shape_fused_start_points(cuda_ok, loc_type, R, n):
    """The fused kernel for 128 input features and bulk-copied R x R records;
    1001 records end in a tile of 105 records whose bytes are not a whole
    number of 16-byte blocks (9x9, 11x11), 1 record likewise."""
    import torch
    rec, para, _ = gen(loc_type, R, 4096, 13 + R)
    d = to_dev(rec)
    feat, scale = qlib.LearnedNet.features(para, d.data_ptr(), rec.shape[0])
    rows = plain_rows(rec, para)
    d_rows = to_dev(rows.astype(np.float32))
    t, v = qlib.LearnedNet.targets(para, d.data_ptr(), d_rows.data_ptr(), scale, rec.shape[0])
    net = qlib.LearnedNet(batch=1024, seed=4, loc_type=loc_type, roi_size=R)
    net.train(feat, t, v, epochs=2, lr=2e-3)
    net.set_fused(True)
    fused = net.start(para, d.data_ptr(), n).cpu().numpy().astype(np.float64)
    net.fused_status()
    net.set_fused(False)
    layered = net.start(para, d.data_ptr(), n).cpu().numpy().astype(np.float64)
    torch.cuda.synchronize()
    sc = scale.cpu().numpy()[:n]
    assert fused.shape[1] == (6 if loc_type == 1 else 5)
    assert np.all(np.isfinite(fused))
    y_o, _ = NO.forward(net.params(), feat[:n].cpu().numpy())
    y_scale = max(1.0, float(np.max(np.abs(y_o))))
    assert_start_close(fused, layered, sc, 2e-3 * y_scale)
    assert_start_close(fused, start_from_y(y_o, sc, R, loc_type), sc, 2e-3 * y_scale)
    net.close()


def test_network_shape_must_match_the_call(cuda_ok):
    rec, para, _ = gen(1, 9, 100, 1)
    net = qlib.LearnedNet(batch=64, seed=1, loc_type=0, roi_size=9)
    ctx = qlib.LocContext(para, capacity=100)
    d = to_dev(rec)
    with pytest.raises(RuntimeError):
        net.localize(ctx, d.data_ptr(), 100, iters=2, bisections=6)
    with pytest.raises(RuntimeError):
        qlib.LearnedNet(batch=64, seed=1, loc_type=1, roi_size=13)
    with pytest.raises(RuntimeError):  # count classes are a GS2D head
        qlib.LearnedNet(batch=64, seed=1, loc_type=1, roi_size=9).set_count_threshold(0.5)
    ctx.close()
    net.close()


def roi_xy(rows, rec, R, sel):
    fx = rows[sel, 1] + R // 2 - rec[sel, R * R].astype(np.float64)
    fy = rows[sel, 2] + R // 2 - rec[sel, R * R + 1].astype(np.float64)
    return fx, fy


@pytest.mark.parametrize("loc_type,R,iters", [(1, 9, 3), (0, 9, 2)])
def test_trained_shape_reaches_plain_rmse(cuda_ok, loc_type, R, iters):
    """Train on 200k ROIs labelled by plain fits; on 40k fresh ROIs, `iters`
    BFGS iterations of 6 line-search steps from the network's start points
    (plus plain refits of the fits the deviance judge rejects) reach the
    position RMSE of plain fits (GS2D 8 iterations, AS3D 11) within 2%, and
    for AS3D the z RMSE within 2%."""
    import torch
    tr, para, _ = gen(loc_type, R, 200_000, 101 + R)
    ev, _, truth = gen(loc_type, R, 40_000, 202 + R)
    n = tr.shape[0]
    d_tr = to_dev(tr)
    ctx_tr = qlib.LocContext(para, capacity=n)
    s = torch.cuda.Stream()
    ctx_tr.localize_device(d_tr.data_ptr(), n, 0, s.cuda_stream)
    s.synchronize()
    feat, scale = qlib.LearnedNet.features(para, d_tr.data_ptr(), n, stream=s.cuda_stream)
    t, v = qlib.LearnedNet.targets(para, d_tr.data_ptr(), ctx_tr.device_rows(), scale, n, stream=s.cuda_stream)
    net = qlib.LearnedNet(batch=4096, seed=5, loc_type=loc_type, roi_size=R)
    losses = net.train(feat, t, v, epochs=8, lr=2e-3, stream=s.cuda_stream)
    assert losses[-1] < 0.5 * losses[0]
    ctx_tr.close()

    m = ev.shape[0]
    d_ev = to_dev(ev)
    ctx = qlib.LocContext(para, capacity=m)
    ctx.localize_device(d_ev.data_ptr(), m, 0, s.cuda_stream)
    plain, _ = ctx.read_rows(s.cuda_stream)
    net.localize(ctx, d_ev.data_ptr(), m, iters=iters, bisections=6, stream=s.cuda_stream)
    learned, _ = ctx.read_rows(s.cuda_stream)
    refits = net.refits(ctx)
    net.fused_status()
    both = (plain[:, 0] > 0) & (learned[:, 0] > 0)
    px, py = roi_xy(plain, ev, R, both)
    lx, ly = roi_xy(learned, ev, R, both)
    tx, ty = truth["x"][both], truth["y"][both]
    r_plain = float(np.sqrt(np.mean((px - tx) ** 2 + (py - ty) ** 2) / 2))
    r_learn = float(np.sqrt(np.mean((lx - tx) ** 2 + (ly - ty) ** 2) / 2))
    msg = "rmse px plain %.5f learned %.5f; refits %d; accepted %.4f / %.4f" % (
        r_plain, r_learn, refits, (plain[:, 0] > 0).mean(), (learned[:, 0] > 0).mean())
    if loc_type == 1:
        z_plain = float(np.sqrt(np.mean((plain[both, 3] - truth["z"][both]) ** 2)))
        z_learn = float(np.sqrt(np.mean((learned[both, 3] - truth["z"][both]) ** 2)))
        msg += "; z rmse nm plain %.2f learned %.2f" % (z_plain, z_learn)
        assert z_learn <= 1.02 * z_plain
    print(msg)
    assert r_learn <= 1.02 * r_plain
    assert refits <= 0.15 * m
    assert (learned[:, 0] > 0).mean() >= (plain[:, 0] > 0).mean() - 0.01
    ctx.close()
    net.close()
