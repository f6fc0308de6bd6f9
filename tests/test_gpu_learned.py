"""Learned start points for GS2D 7x7 fits (qcs_learned_*, qcs_fit_from_start_device).

The network's features, targets, forward pass and parameter gradient are
checked against the numpy restatement in oracle/qcs_net_oracle.py (GEMM
operands rounded to bfloat16 like the tensor-core kernels; float64
accumulation there, float32 here).  Then a network trained on the GPU is
shown to buy what it is for: fits from its start points with 3 BFGS
iterations (plus plain refits of the few that fail the goodness-of-fit
judge) reach the RMSE of plain 8-iteration fits, while 3 iterations from the
plain centre / edge-mean start do not.
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


def plain_rows(rec, para):
    ctx = qlib.LocContext(para, capacity=rec.shape[0])
    rows, _ = ctx.localize(rec)
    ctx.close()
    return rows


def to_dev(a, dtype=None):
    import torch
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint16:
        a = a.view(np.int16)
    return torch.from_numpy(a).cuda()


def test_features_and_targets_match_oracle(cuda_ok):
    rec, para, _ = synth.gs2d_rois(3000, seed=11)
    d = to_dev(rec)
    n = rec.shape[0]
    feat, scale = qlib.LearnedNet.features(para, d.data_ptr(), n)
    f_o, s_o = NO.features(rec, para.Offset, para.KAdc)
    np.testing.assert_allclose(feat.cpu().numpy(), f_o, rtol=2e-6, atol=2e-6)
    np.testing.assert_array_equal(scale.cpu().numpy(), s_o)
    rows = plain_rows(rec, para)
    d_rows = to_dev(rows.astype(np.float32))
    t, v = qlib.LearnedNet.targets(para, d.data_ptr(), d_rows.data_ptr(), scale, n)
    t_o, v_o = NO.targets(rec, rows, s_o, para.QE)
    np.testing.assert_array_equal(v.cpu().numpy(), v_o)
    np.testing.assert_allclose(t.cpu().numpy(), t_o, rtol=1e-5, atol=1e-5)


def test_forward_and_gradient_match_oracle(cuda_ok):
    rec, para, _ = synth.gs2d_rois(512, seed=12)
    d = to_dev(rec)
    n = rec.shape[0]
    feat, scale = qlib.LearnedNet.features(para, d.data_ptr(), n)
    rows = plain_rows(rec, para)
    d_rows = to_dev(rows.astype(np.float32))
    t, v = qlib.LearnedNet.targets(para, d.data_ptr(), d_rows.data_ptr(), scale, n)
    net = qlib.LearnedNet(batch=512, seed=3)
    params = net.params()
    y = net.forward(feat).cpu().numpy()
    loss = net.gradient(feat, t, v)
    g = net.grads()
    loss_o, g_o, y_o = NO.loss_and_grad(params, feat.cpu().numpy(), t.cpu().numpy(), v.cpu().numpy())
    assert np.max(np.abs(y - y_o)) <= 2e-3 * max(1.0, np.max(np.abs(y_o)))
    assert abs(loss - loss_o) <= 2e-3 * abs(loss_o)
    # per parameter block: relative error of the gradient
    o = 0
    for size in (64 * 128, 128, 128 * 128, 128, 128 * 8, 8):
        a, b = g[o:o + size], g_o[o:o + size]
        o += size
        assert np.linalg.norm(a - b) <= 2e-2 * np.linalg.norm(b) + 1e-7, (size, np.linalg.norm(a - b), np.linalg.norm(b))
    net.close()


def test_fused_start_points_misaligned_records(cuda_ok):
    """Records not on a 16-byte boundary cannot be bulk-copied: the fused kernel
    then loads each record directly and gives the same start points."""
    import torch
    rec, para, _ = synth.gs2d_rois(3000, seed=14)
    n = rec.shape[0]
    d = to_dev(rec)
    buf = torch.zeros(n * rec.shape[1] + 4, dtype=torch.int16, device="cuda")
    buf[4:] = d.reshape(-1)
    net = qlib.LearnedNet(batch=512, seed=8)
    a = net.start(para, d.data_ptr(), n).cpu().numpy()
    b = net.start(para, buf.data_ptr() + 8, n).cpu().numpy()
    net.fused_status()
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    net.close()


def start_from_y(y, scale):
    """The start-point transform of the network outputs (clamps as in qcs_learned.cu start_kernel)."""
    lo, rng = scale[:, 0].astype(np.float64), scale[:, 1].astype(np.float64)
    return np.stack([rng * np.exp(np.clip(y[:, 3], -6, 3)), NO.CENTRE + np.clip(y[:, 0], -1.5, 1.5),
                     NO.CENTRE + np.clip(y[:, 1], -1.5, 1.5), np.clip(NO.SIGMA0 + y[:, 2], 0.6, 3.0),
                     np.maximum(lo + rng * y[:, 4], 1.0)], 1)


def assert_start_close(a, b, scale, tol):
    """Start points agree to `tol` in network-output units: relative for the
    peak (exp of an output), absolute for x, y, sigma, background / range."""
    rng = scale[:, 1].astype(np.float64)
    assert np.max(np.abs(np.log(a[:, 0] / b[:, 0]))) <= tol
    assert np.max(np.abs(a[:, 1:4] - b[:, 1:4])) <= tol
    assert np.max(np.abs(a[:, 4] - b[:, 4]) / rng) <= tol


@pytest.mark.parametrize("n", [1, 1000, 100_000])
def test_fused_tensor_core_start_points(cuda_ok, n):
    """The fused tcgen05 inference kernel (features, three BF16 GEMMs with
    FP32 accumulation in tensor memory, start transform, one launch) against
    the layer-by-layer path and against the numpy forward pass: the ragged
    last 128-ROI tile, a single ROI, and more tiles than resident CTAs.  The
    network is trained briefly so that its outputs are not near zero."""
    import torch
    rec, para, _ = synth.gs2d_rois(max(n, 4096), seed=13)
    d = to_dev(rec)
    feat, scale = qlib.LearnedNet.features(para, d.data_ptr(), rec.shape[0])
    rows = plain_rows(rec, para)
    d_rows = to_dev(rows.astype(np.float32))
    t, v = qlib.LearnedNet.targets(para, d.data_ptr(), d_rows.data_ptr(), scale, rec.shape[0])
    net = qlib.LearnedNet(batch=1024, seed=4)
    net.train(feat, t, v, epochs=2, lr=2e-3)
    net.set_fused(True)
    fused = net.start(para, d.data_ptr(), n).cpu().numpy().astype(np.float64)
    net.fused_status()
    net.set_fused(False)
    layered = net.start(para, d.data_ptr(), n).cpu().numpy().astype(np.float64)
    torch.cuda.synchronize()
    sc = scale.cpu().numpy()[:n]
    assert np.all(np.isfinite(fused))
    y_scale = max(1.0, float(np.max(np.abs(NO.forward(net.params(), feat[:min(n, 2048)].cpu().numpy())[0]))))
    assert_start_close(fused, layered, sc, 2e-3 * y_scale)
    k = min(n, 2048)
    y_o, _ = NO.forward(net.params(), feat[:k].cpu().numpy())
    assert_start_close(fused[:k], start_from_y(y_o, sc[:k]), sc[:k], 2e-3 * y_scale)
    net.close()


def rmse_xy(rows, rec, truth, sel):
    """RMSE per axis (px) of the fitted centres in ROI coordinates: the row's
    x is fit - R/2 + header x (header word 0 / 1 of the record)."""
    R = 7
    fx = rows[sel, 1] + R // 2 - rec[sel, R * R].astype(np.float64)
    fy = rows[sel, 2] + R // 2 - rec[sel, R * R + 1].astype(np.float64)
    return float(np.sqrt(np.mean((fx - truth["x"][sel]) ** 2 + (fy - truth["y"][sel]) ** 2) / 2))


def naive_start(rec, para):
    """The plain fit's own pre-estimate (centre, edge-mean background, sigma 1.3)."""
    e = np.maximum((rec[:, :49].astype(np.float32) - para.Offset) * para.KAdc, 1.0).reshape(-1, 7, 7)
    m1 = np.minimum(e[:, 0, :].mean(1) * 7, e[:, 6, :].mean(1) * 7)
    m3 = np.minimum(e[:, :, 0].mean(1) * 7, e[:, :, 6].mean(1) * 7)
    bkg = (m1 + m3) / 2 / 7
    peak = np.maximum(e[:, 3, 3] - bkg, 1.0)
    st = np.stack([peak, np.full_like(peak, 3.5), np.full_like(peak, 3.5), np.full_like(peak, 1.3), bkg], 1)
    return np.ascontiguousarray(st, np.float32)


def test_refits_reproduce_plain_rows(cuda_ok):
    """With a deviance bound no fit meets, every record is refitted plainly
    (group kernel on the side stream, CRLB of the refit queue there, the
    main-stream CRLB skipping those rows): the rows, CRLB columns included,
    equal the plain localization's bit for bit."""
    import ctypes as C
    import torch
    rec, para, _ = synth.gs2d_rois(20_000, seed=31)
    n = rec.shape[0]
    d = to_dev(rec)
    ctx = qlib.LocContext(para, capacity=n)
    s = torch.cuda.Stream()
    ctx.localize_device(d.data_ptr(), n, 0, s.cuda_stream)
    plain, _ = ctx.read_rows(s.cuda_stream)
    st = to_dev(naive_start(rec, para))
    qlib.fit_from_start(ctx, d.data_ptr(), n, st.data_ptr(), iters=2, dev_th=1e-6, stream=s.cuda_stream)
    refit, _ = ctx.read_rows(s.cuda_stream)
    k = C.c_int(0)
    qlib.check(qlib.load().qcs_learned_refit_num(ctx.h, C.byref(k)))
    assert k.value == n
    np.testing.assert_array_equal(refit.view(np.uint32), plain.view(np.uint32))
    ctx.close()


def rmse_photons(rows, truth, sel):
    return float(np.sqrt(np.mean((rows[sel, 6] / truth["photons"][sel] - 1) ** 2)))


@pytest.mark.parametrize("bisections", [11, 6])
def test_trained_start_points_reach_plain_rmse_with_fewer_iterations(cuda_ok, bisections):
    """Train on 200k ROIs labelled by plain fits; on 50k fresh ROIs, 2 BFGS
    iterations (11 or 6 line-search steps) from the network's start points (plus plain refits of the
    fits the deviance judge rejects) match plain 8-iteration fits in position
    RMSE and beat them in photon RMSE, while 2 iterations from the plain
    centre / edge-mean start do not reach the plain RMSE."""
    import torch
    tr, para, _ = synth.gs2d_rois(200_000, seed=101)
    ev, _, truth = synth.gs2d_rois(50_000, seed=202)
    n = tr.shape[0]
    d_tr = to_dev(tr)
    feat, scale = qlib.LearnedNet.features(para, d_tr.data_ptr(), n)
    rows_tr = plain_rows(tr, para)
    d_rows = to_dev(rows_tr.astype(np.float32))
    t, v = qlib.LearnedNet.targets(para, d_tr.data_ptr(), d_rows.data_ptr(), scale, n)
    net = qlib.LearnedNet(batch=4096, seed=5)
    losses = net.train(feat, t, v, epochs=8, lr=2e-3)
    assert losses[-1] < 0.5 * losses[0]

    m = ev.shape[0]
    d_ev = to_dev(ev)
    ctx = qlib.LocContext(para, capacity=m)
    s = torch.cuda.Stream()
    ctx.localize_device(d_ev.data_ptr(), m, 0, s.cuda_stream)
    plain, _ = ctx.read_rows(s.cuda_stream)
    net.localize(ctx, d_ev.data_ptr(), m, iters=2, bisections=bisections, stream=s.cuda_stream)
    learned, _ = ctx.read_rows(s.cuda_stream)
    refits = net.refits(ctx)
    d_start = to_dev(naive_start(ev, para))
    qlib.fit_from_start(ctx, d_ev.data_ptr(), m, d_start.data_ptr(), iters=2, bisections=bisections,
                        stream=s.cuda_stream)
    naive, _ = ctx.read_rows(s.cuda_stream)
    both = (plain[:, 0] > 0) & (learned[:, 0] > 0) & (naive[:, 0] > 0)
    r_plain, r_learn, r_naive = (rmse_xy(plain, ev, truth, both), rmse_xy(learned, ev, truth, both),
                                 rmse_xy(naive, ev, truth, both))
    p_plain, p_learn = rmse_photons(plain, truth, both), rmse_photons(learned, truth, both)
    print("rmse px plain %.5f learned %.5f naive %.5f; photons plain %.4f learned %.4f; refits %d" % (
        r_plain, r_learn, r_naive, p_plain, p_learn, refits))
    assert r_learn <= 1.02 * r_plain
    assert p_learn <= p_plain
    assert r_naive > 1.05 * r_plain
    assert refits <= 0.10 * m
    assert (learned[:, 0] > 0).mean() >= (plain[:, 0] > 0).mean() - 0.005
    # without the plain refits (qcs_learned_set_single_refits): no refit pass, the same accuracy
    net.set_single_refits(False)
    net.localize(ctx, d_ev.data_ptr(), m, iters=2, bisections=bisections, stream=s.cuda_stream)
    nr, _ = ctx.read_rows(s.cuda_stream)
    assert net.refits(ctx) == 0
    both_nr = (plain[:, 0] > 0) & (nr[:, 0] > 0)
    assert rmse_xy(nr, ev, truth, both_nr) <= 1.02 * rmse_xy(plain, ev, truth, both_nr)
    assert (nr[:, 0] > 0).mean() >= (plain[:, 0] > 0).mean() - 0.005
    # rows the default call did not refit are the no-refit call's bit for bit
    same = (learned[:, 0] > 0) & (nr[:, 0] > 0)
    assert np.mean(np.all(learned[same].view(np.uint32) == nr[same].view(np.uint32), axis=1)) >= 1.0 - refits / m
    net.set_single_refits(True)
    ctx.close()
    net.close()
