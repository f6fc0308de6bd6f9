"""Convolutional start-point network (QCS_LEARNED_ARCH_CONV: 3x3 conv 32 ->
3x3 conv 64 -> FC 256 -> the MLP's eight outputs).

Forward pass, loss and parameter gradient of the GPU training path (im2col
and tcgen05 GEMMs) against the numpy restatement in
oracle/qcs_net_oracle.py (conv_loss_and_grad, itself checked by finite
differences in tests/test_oracle_convnet.py); the two-kernel tcgen05
inference (conv kernel on a padded row grid, FC + head kernel on a bulk-copy
ring) against the layer-by-layer path and the numpy forward pass, including
a call of more than one 65,536-record chunk; and a trained network's fits
against the plain fits.
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
    """The start transform of the network outputs (start_from_outputs in qcs_learned.h)."""
    lo, rng = scale[:, 0].astype(np.float64), scale[:, 1].astype(np.float64)
    win, smax = (2.5, 4.0) if loc_type == 1 else (1.5, 3.0)
    cols = [rng * np.exp(np.clip(y[:, 3], -6, 3)), R / 2.0 + np.clip(y[:, 0], -win, win),
            R / 2.0 + np.clip(y[:, 1], -win, win), np.clip(NO.SIGMA0 + y[:, 2], 0.6, smax)]
    if loc_type == 1:
        cols.append(np.clip(NO.SIGMA0 + y[:, 5], 0.6, smax))
    cols.append(np.maximum(lo + rng * y[:, 4], 1.0))
    return np.stack(cols, 1)


def assert_start_close(a, b, scale, tol):
    rng = scale[:, 1].astype(np.float64)
    assert np.max(np.abs(np.log(a[:, 0] / b[:, 0]))) <= tol
    assert np.max(np.abs(a[:, 1:-1] - b[:, 1:-1])) <= tol
    assert np.max(np.abs(a[:, -1] - b[:, -1]) / rng) <= tol


def data(loc_type, R, n, seed):
    rec, para, truth = gen(loc_type, R, n, seed)
    d = to_dev(rec)
    feat, scale = qlib.LearnedNet.features(para, d.data_ptr(), n)
    rows = plain_rows(rec, para)
    d_rows = to_dev(rows.astype(np.float32))  # kept alive while the kernel reads it
    t, v = qlib.LearnedNet.targets(para, d.data_ptr(), d_rows.data_ptr(), scale, n)
    return rec, para, truth, d, feat, scale, t, v, d_rows


def blocks(R):
    return (9 * 32, 32, 288 * 64, 64, (R * R * 64 + 2) * 256, 256, 256 * 8, 8)


@pytest.mark.parametrize("loc_type,R", [(0, 7), (0, 11), (1, 9)])
def test_conv_forward_and_gradient_match_oracle(cuda_ok, loc_type, R):
    import torch
    n = 256
    rec, para, _, d, feat, scale, t, v, _keep = data(loc_type, R, n, 40 + R)
    net = qlib.LearnedNet(batch=n, seed=3, loc_type=loc_type, roi_size=R, arch="conv")
    assert net.n_params == NO.conv_param_count(R)
    params = net.params()
    y = net.forward(feat).cpu().numpy()
    classes = None
    if loc_type == 0:
        classes = torch.from_numpy(np.random.default_rng(R).integers(-1, 3, n).astype(np.float32)).cuda()
    loss = net.gradient(feat, t, v, classes=classes)
    g = net.grads()
    loss_o, g_o, y_o = NO.conv_loss_and_grad(params, feat.cpu().numpy(), t.cpu().numpy(), v.cpu().numpy(), R,
                                             classes=None if classes is None else classes.cpu().numpy())
    assert np.max(np.abs(y - y_o)) <= 2e-3 * max(1.0, np.max(np.abs(y_o)))
    assert abs(loss - loss_o) <= 2e-3 * abs(loss_o)
    o = 0
    for size in blocks(R):
        a, b = g[o:o + size], g_o[o:o + size]
        o += size
        assert np.linalg.norm(a - b) <= 2e-2 * np.linalg.norm(b) + 1e-7, (size, np.linalg.norm(a - b),
                                                                          np.linalg.norm(b))
    net.close()


@pytest.mark.parametrize("loc_type,R,n", [(0, 7, 1), (0, 7, 1001), (0, 9, 1001), (0, 11, 1001), (1, 9, 1001),
                                          (0, 7, 70_000)])
def test_conv_tensor_core_start_points(cuda_ok, loc_type, R, n):
    """The two inference kernels against the layer-by-layer path (all n) and
    the numpy forward pass (the first 1024): a single record, ragged last
    groups and tiles, and a call over two chunks.  The network is trained
    briefly so that its outputs are not near zero."""
    m = max(n, 4096)
    rec, para, _, d, feat, scale, t, v, _keep = data(loc_type, R, m, 60 + R)
    net = qlib.LearnedNet(batch=1024, seed=4, loc_type=loc_type, roi_size=R, arch="conv")
    net.train(feat[:4096], t[:4096], v[:4096], epochs=2, lr=1e-3)
    net.set_fused(True)
    fused = net.start(para, d.data_ptr(), n).cpu().numpy().astype(np.float64)
    net.fused_status()
    net.set_fused(False)
    layered = net.start(para, d.data_ptr(), n).cpu().numpy().astype(np.float64)
    sc = scale.cpu().numpy()[:n]
    assert np.all(np.isfinite(fused))
    k = min(n, 1024)
    y_o, _ = NO.conv_forward(net.params(), feat[:k].cpu().numpy(), R)
    y_scale = max(1.0, float(np.max(np.abs(y_o))))
    assert_start_close(fused, layered, sc, 2e-3 * y_scale)
    assert_start_close(fused[:k], start_from_y(y_o, sc[:k], R, loc_type), sc[:k], 2e-3 * y_scale)
    net.close()


def test_conv_network_localize_equals_fit_from_its_start_points(cuda_ok):
    """The learned localization call with a conv network is the fit from that
    network's start points: its rows equal, bit for bit, those of
    qcs_fit_from_start_classes_device given the same start points."""
    import torch
    n = 20_000
    rec, para, _, d, feat, scale, t, v, _keep = data(0, 7, n, 71)
    net = qlib.LearnedNet(batch=4096, seed=4, arch="conv")
    net.train(feat, t, v, epochs=2, lr=1e-3)
    s = torch.cuda.Stream()
    st = net.start(para, d.data_ptr(), n, stream=s.cuda_stream)
    s.synchronize()
    ctx = qlib.LocContext(para, capacity=n)
    net.localize(ctx, d.data_ptr(), n, iters=2, bisections=6, stream=s.cuda_stream)
    a, ra = ctx.read_rows(s.cuda_stream)
    qlib.fit_from_start(ctx, d.data_ptr(), n, st.data_ptr(), iters=2, bisections=6, stream=s.cuda_stream)
    b, rb = ctx.read_rows(s.cuda_stream)
    net.fused_status()
    assert (a[:, 0] > 0).mean() > 0.9
    np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32))
    np.testing.assert_array_equal(ra, rb)
    ctx.close()
    net.close()


@pytest.mark.parametrize("arch,fused", [("conv", True), ("conv", False), ("mlp", True), ("mlp", False)])
def test_learned_calls_on_several_streams(cuda_ok, arch, fused):
    """One network used by three contexts on three streams at once (calls in
    flight together) gives every call the rows it gives alone: the network's
    own inference buffers are handed from call to call in stream order."""
    import torch
    n = 60_000
    rec, para, _, d, feat, scale, t, v, _keep = data(0, 7, 3 * n, 72)
    net = qlib.LearnedNet(batch=4096, seed=4, arch=arch)
    net.train(feat[:20_000], t[:20_000], v[:20_000], epochs=2, lr=1e-3)
    net.set_fused(fused)
    rb = 7 * 8 * 2
    streams = [torch.cuda.Stream() for _ in range(3)]
    ctxs = [qlib.LocContext(para, capacity=n) for _ in range(3)]
    alone = []
    for j in range(3):
        net.localize(ctxs[0], d.data_ptr() + j * n * rb, n, iters=2, bisections=6, stream=streams[0].cuda_stream)
        alone.append(ctxs[0].read_rows(streams[0].cuda_stream)[0])
    torch.cuda.synchronize()
    for rep in range(2):
        for j in range(3):
            net.localize(ctxs[j], d.data_ptr() + j * n * rb, n, iters=2, bisections=6, stream=streams[j].cuda_stream)
        for j in range(3):
            got = ctxs[j].read_rows(streams[j].cuda_stream)[0]
            np.testing.assert_array_equal(got.view(np.uint32), alone[j].view(np.uint32))
    net.fused_status()
    for c in ctxs:
        c.close()
    net.close()
