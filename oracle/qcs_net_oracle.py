"""TEST INFRASTRUCTURE ONLY -- numpy restatement of the learned start-point
network of qc-storm_b200/csrc/qcs_learned.cu (features, targets, forward pass,
masked weighted MSE plus the emitter-count cross-entropy and its gradient,
the class rule), used by the tests to check the GPU kernels' forward outputs,
gradients and classes.  The network has no counterpart in
the reference; its definition is the one in qcs_learned.cu / qcs_learned.h.

GEMM operands are rounded to bfloat16 as the tensor-core kernels round them;
products are accumulated in float64 here (float32 on the GPU), so agreement
is to accumulation rounding, not bit for bit.
"""
import numpy as np

R = 7
PIX = R * R
WHOLE = R * (R + 1)
HALF = R // 2
CENTRE = R / 2.0
SIGMA0 = 1.3
N_IN, N_HID, N_OUT, N_USED = 64, 128, 8, 5
TARGET_WEIGHT = np.array([4.0, 4.0, 1.0, 1.0, 1.0])
COUNT0, CLASSES, COUNT_WEIGHT = 5, 3, 0.5  # outputs 5..7: emitter-count logits
N_PARAMS = N_IN * N_HID + N_HID + N_HID * N_HID + N_HID + N_HID * N_OUT + N_OUT


def bf16(a):
    """Round float32 values to bfloat16 (round to nearest even), kept as float64."""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    rounded = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return rounded.astype(np.uint32).view(np.float32).astype(np.float64)


def split_params(p):
    p = np.asarray(p, np.float64)
    o = 0
    out = []
    for shape in ((N_IN, N_HID), (N_HID,), (N_HID, N_HID), (N_HID,), (N_HID, N_OUT), (N_OUT,)):
        size = int(np.prod(shape))
        out.append(p[o:o + size].reshape(shape))
        o += size
    return out


def features(rois, offset, kadc):
    e = np.maximum((rois[:, :PIX].astype(np.float32) - np.float32(offset)) * np.float32(kadc), np.float32(1.0))
    lo = e.min(axis=1)
    rng = np.maximum(e.max(axis=1) - lo, np.float32(1.0))
    f = np.zeros((rois.shape[0], N_IN), np.float32)
    f[:, :PIX] = (e - lo[:, None]) * (np.float32(1.0) / rng)[:, None]
    f[:, PIX] = np.log(rng) * np.float32(0.125)
    f[:, PIX + 1] = np.log(lo) * np.float32(0.125)
    return f, np.stack([lo, rng], axis=1)


def targets(rois, rows, scale, qe):
    lo, rng = scale[:, 0], scale[:, 1]
    ok = (rows[:, 0] > 0) & (rows[:, 4] > 0)
    t = np.zeros((rows.shape[0], N_USED), np.float32)
    hx = rois[:, PIX].astype(np.float32)
    hy = rois[:, PIX + 1].astype(np.float32)
    t[:, 0] = rows[:, 1] + HALF - hx - CENTRE
    t[:, 1] = rows[:, 2] + HALF - hy - CENTRE
    t[:, 2] = rows[:, 4] - SIGMA0
    t[:, 3] = np.log(np.maximum(rows[:, 0] * qe, 1e-3) / rng)
    t[:, 4] = (rows[:, 7] * qe - lo) / rng
    t[~ok] = 0
    return t, ok.astype(np.float32)


def forward(params, x):
    W1, b1, W2, b2, W3, b3 = split_params(params)
    z1 = bf16(x) @ bf16(W1) + b1
    a1 = np.maximum(z1, 0)
    z2 = bf16(a1) @ bf16(W2) + b2
    a2 = np.maximum(z2, 0)
    y = bf16(a2) @ bf16(W3) + b3
    return y, (x, z1, a1, z2, a2)


def count_class(logits, th):
    """Emitter-count class per row of the three logits: 2 when p2 >= th, else
    1 when p1 + p2 >= th, else 0 (float32 softmax numerators, as the kernels)."""
    lg = np.asarray(logits, np.float32)
    e = np.exp(lg - lg.max(axis=1, keepdims=True))
    s = e.sum(axis=1)
    th = np.float32(th)
    return np.where(e[:, 2] >= th * s, 2, np.where(e[:, 1] + e[:, 2] >= th * s, 1, 0)).astype(np.uint8)


def loss_and_grad(params, x, t, valid, classes=None):
    """Mean over the batch of sum_j w_j (y_j - t_j)^2 * valid plus, for rows
    with a class label c >= 0, COUNT_WEIGHT * (-log softmax(logits)[c]); and
    its gradient."""
    W1, b1, W2, b2, W3, b3 = split_params(params)
    y, (x, z1, a1, z2, a2) = forward(params, x)
    n = x.shape[0]
    e = y[:, :N_USED] - t
    loss = float(np.sum(TARGET_WEIGHT * e * e * valid[:, None]) / n)
    dy = np.zeros_like(y)
    dy[:, :N_USED] = 2.0 * TARGET_WEIGHT * e * valid[:, None] / n
    if classes is not None:
        c = np.asarray(classes).astype(np.int64)
        lab = c >= 0
        lg = y[:, COUNT0:COUNT0 + CLASSES]
        m = lg.max(axis=1, keepdims=True)
        p = np.exp(lg - m)
        p /= p.sum(axis=1, keepdims=True)
        rows = np.nonzero(lab)[0]
        loss += float(COUNT_WEIGHT * np.sum(-np.log(p[rows, c[rows]])) / n)
        onehot = np.zeros_like(p)
        onehot[rows, c[rows]] = 1.0
        dy[:, COUNT0:COUNT0 + CLASSES] = COUNT_WEIGHT * (p - onehot) * lab[:, None] / n
    gW3 = bf16(a2).T @ bf16(dy)
    gb3 = dy.sum(axis=0)
    d2 = bf16(dy) @ bf16(W3).T
    d2 = d2 * (z2 > 0)
    gW2 = bf16(a1).T @ bf16(d2)
    gb2 = d2.sum(axis=0)
    d1 = bf16(d2) @ bf16(W2).T
    d1 = d1 * (z1 > 0)
    gW1 = bf16(x).T @ bf16(d1)
    gb1 = d1.sum(axis=0)
    grad = np.concatenate([g.ravel() for g in (gW1, gb1, gW2, gb2, gW3, gb3)])
    return loss, grad, y
