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
N_IN, N_HID, N_OUT, N_USED = 64, 128, 8, 5   # the GS2D 7x7 network
TARGET_WEIGHT = np.array([4.0, 4.0, 1.0, 1.0, 1.0, 1.0])  # GS2D uses the first 5, AS3D all 6
TARGET_WEIGHT_2E = np.array([4.0, 4.0, 4.0, 4.0, 1.0, 1.0, 1.0, 1.0])  # the two-emitter start points
TARGET_WEIGHT_3E = np.array([4.0, 4.0, 4.0, 4.0, 4.0, 4.0, 1.0, 1.0, 1.0, 1.0, 1.0])  # the three-emitter ones
LEARNED_2E = 16  # network kind of the two-emitter start points (QCS_LEARNED_GS2D_2E)
LEARNED_3E = 17  # network kind of the three-emitter start points (QCS_LEARNED_GS2D_3E; 16 outputs)


def in_width(r):
    """Input width of the network for r x r ROIs (r*r pixels + 2 scale features, padded)."""
    return 64 if r * r + 2 <= 64 else 128


def used_outputs(loc_type):
    return 11 if loc_type == LEARNED_3E else (8 if loc_type == LEARNED_2E else (6 if loc_type == 1 else 5))


def out_width(loc_type):
    return 16 if loc_type == LEARNED_3E else N_OUT


def start_points_3e(y, lo, rng, r):
    """Three-emitter start points (peak, x, y of emitters 0..2, sigma,
    background) from outputs y [n, 16] and the ROI scales, as the kernels map
    them (positions held a pixel inside the ROI's edge)."""
    y = np.asarray(y, np.float64)
    c, w2 = r / 2.0, r / 2.0 - 1.0
    st = np.zeros((y.shape[0], 11))
    for e in range(3):
        st[:, 3 * e] = rng * np.exp(np.clip(y[:, 6 + e], -6, 3))
        st[:, 3 * e + 1] = c + np.clip(y[:, 2 * e], -w2, w2)
        st[:, 3 * e + 2] = c + np.clip(y[:, 2 * e + 1], -w2, w2)
    st[:, 9] = np.clip(SIGMA0 + y[:, 9], 0.6, 3.0)
    st[:, 10] = np.maximum(lo + rng * y[:, 10], 1.0)
    return st


def start_points_2e(y, lo, rng, r):
    """Two-emitter start points (peak0, x0, y0, peak1, x1, y1, sigma,
    background) from outputs y [n, 8] and the ROI scales, as the kernels map
    them (positions held a pixel inside the ROI's edge)."""
    y = np.asarray(y, np.float64)
    c, w2 = r / 2.0, r / 2.0 - 1.0
    st = np.zeros((y.shape[0], 8))
    st[:, 0] = rng * np.exp(np.clip(y[:, 4], -6, 3))
    st[:, 1] = c + np.clip(y[:, 0], -w2, w2)
    st[:, 2] = c + np.clip(y[:, 1], -w2, w2)
    st[:, 3] = rng * np.exp(np.clip(y[:, 5], -6, 3))
    st[:, 4] = c + np.clip(y[:, 2], -w2, w2)
    st[:, 5] = c + np.clip(y[:, 3], -w2, w2)
    st[:, 6] = np.clip(SIGMA0 + y[:, 6], 0.6, 3.0)
    st[:, 7] = np.maximum(lo + rng * y[:, 7], 1.0)
    return st


def param_count(n_in, n_out=None):
    n_out = N_OUT if n_out is None else n_out
    return n_in * N_HID + N_HID + N_HID * N_HID + N_HID + N_HID * n_out + n_out
COUNT0, CLASSES, COUNT_WEIGHT = 5, 3, 0.5  # outputs 5..7: emitter-count logits
N_PARAMS = N_IN * N_HID + N_HID + N_HID * N_HID + N_HID + N_HID * N_OUT + N_OUT


def bf16(a):
    """Round float32 values to bfloat16 (round to nearest even), kept as float64."""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    rounded = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return rounded.astype(np.uint32).view(np.float32).astype(np.float64)


def split_params(p, n_out=None):
    n_out = N_OUT if n_out is None else n_out
    p = np.asarray(p, np.float64)
    n_in = (p.size - param_count(0, n_out)) // N_HID
    o = 0
    out = []
    for shape in ((n_in, N_HID), (N_HID,), (N_HID, N_HID), (N_HID,), (N_HID, n_out), (n_out,)):
        size = int(np.prod(shape))
        out.append(p[o:o + size].reshape(shape))
        o += size
    return out


def features(rois, offset, kadc, r=R):
    pix = r * r
    e = np.maximum((rois[:, :pix].astype(np.float32) - np.float32(offset)) * np.float32(kadc), np.float32(1.0))
    lo = e.min(axis=1)
    rng = np.maximum(e.max(axis=1) - lo, np.float32(1.0))
    f = np.zeros((rois.shape[0], in_width(r)), np.float32)
    f[:, :pix] = (e - lo[:, None]) * (np.float32(1.0) / rng)[:, None]
    f[:, pix] = np.log(rng) * np.float32(0.125)
    f[:, pix + 1] = np.log(lo) * np.float32(0.125)
    return f, np.stack([lo, rng], axis=1)


def targets(rois, rows, scale, qe, r=R, loc_type=0):
    """GS2D: dx, dy, sigma - 1.3, log(peak / range), (bkg - min) / range; AS3D
    adds sigma_y - 1.3 (the row's sigma_x, sigma_y in columns 4, 5)."""
    pix = r * r
    lo, rng = scale[:, 0], scale[:, 1]
    ok = (rows[:, 0] > 0) & (rows[:, 4] > 0)
    t = np.zeros((rows.shape[0], used_outputs(loc_type)), np.float32)
    hx = rois[:, pix].astype(np.float32)
    hy = rois[:, pix + 1].astype(np.float32)
    t[:, 0] = rows[:, 1] + r // 2 - hx - r / 2.0
    t[:, 1] = rows[:, 2] + r // 2 - hy - r / 2.0
    t[:, 2] = rows[:, 4] - SIGMA0
    t[:, 3] = np.log(np.maximum(rows[:, 0] * qe, 1e-3) / rng)
    t[:, 4] = (rows[:, 7] * qe - lo) / rng
    if loc_type == 1:
        t[:, 5] = rows[:, 5] - SIGMA0
    t[~ok] = 0
    return t, ok.astype(np.float32)


def forward(params, x, n_out=None):
    W1, b1, W2, b2, W3, b3 = split_params(params, n_out)
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


def loss_and_grad(params, x, t, valid, classes=None, n_out=None):
    """Mean over the batch of sum_j w_j (y_j - t_j)^2 * valid plus, for rows
    with a class label c >= 0, COUNT_WEIGHT * (-log softmax(logits)[c]); and
    its gradient."""
    W1, b1, W2, b2, W3, b3 = split_params(params, n_out)
    y, (x, z1, a1, z2, a2) = forward(params, x, n_out)
    n = x.shape[0]
    nu = t.shape[1]
    e = y[:, :nu] - t
    tw = TARGET_WEIGHT_3E if nu == 11 else (TARGET_WEIGHT_2E if nu == 8 else TARGET_WEIGHT[:nu])
    loss = float(np.sum(tw * e * e * valid[:, None]) / n)
    dy = np.zeros_like(y)
    dy[:, :nu] = 2.0 * tw * e * valid[:, None] / n
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


# ---------------------------------------------------------------- conv net
# The convolutional start-point network (QCS_LEARNED_ARCH_CONV in
# qc-storm_b200/csrc/qcs_convnet.cu): the R x R scaled pixels (the first R*R
# features) -> 3x3 conv, 32 channels, zero 'same' padding, ReLU -> 3x3 conv,
# 64 channels, ReLU -> fully connected 256 over the flattened map (position
# major, channel minor) and the two scale features, ReLU -> 8 outputs (the
# MLP's outputs).  Parameters, row-major [in][out]: W1 [9][32] (tap t = 3 *
# (dy + 1) + (dx + 1)), b1, W2 [9 * 32][64] (row t * 32 + input channel), b2,
# W3 [R*R*64 + 2][256], b3, W4 [256][8], b4.
CONV_C1, CONV_C2, CONV_FC = 32, 64, 256


def conv_param_count(r):
    return 9 * CONV_C1 + CONV_C1 + 9 * CONV_C1 * CONV_C2 + CONV_C2 + (r * r * CONV_C2 + 2) * CONV_FC + CONV_FC + \
        CONV_FC * N_OUT + N_OUT


def conv_split_params(p, r):
    p = np.asarray(p, np.float64)
    shapes = ((9, CONV_C1), (CONV_C1,), (9 * CONV_C1, CONV_C2), (CONV_C2,), (r * r * CONV_C2 + 2, CONV_FC),
              (CONV_FC,), (CONV_FC, N_OUT), (N_OUT,))
    out, o = [], 0
    for shape in shapes:
        size = int(np.prod(shape))
        out.append(p[o:o + size].reshape(shape))
        o += size
    assert o == p.size
    return out


def im2col(a, r):
    """[n, r, r, c] -> [n * r * r, 9 * c]: for each position the 3x3
    neighbourhood (tap-major, channel-minor), zeros outside the ROI."""
    n, c = a.shape[0], a.shape[3]
    pad = np.zeros((n, r + 2, r + 2, c))
    pad[:, 1:-1, 1:-1] = a
    cols = [pad[:, dy:dy + r, dx:dx + r, :] for dy in range(3) for dx in range(3)]
    return np.concatenate(cols, axis=3).reshape(n * r * r, 9 * c)


def col2im(d, n, r, c):
    """Adjoint of im2col: [n * r * r, 9 * c] -> [n * r * r, c]."""
    d = d.reshape(n, r, r, 9, c)
    pad = np.zeros((n, r + 2, r + 2, c))
    for dy in range(3):
        for dx in range(3):
            pad[:, dy:dy + r, dx:dx + r, :] += d[:, :, :, dy * 3 + dx, :]
    return pad[:, 1:-1, 1:-1, :].reshape(n * r * r, c)


def conv_forward(params, x, r, exact=False):
    """Outputs [n, 8] of feature rows x (in_width(r) wide).  GEMM operands are
    rounded to bfloat16 as the GPU rounds them, unless exact."""
    rb = (lambda a: np.asarray(a, np.float64)) if exact else bf16
    W1, b1, W2, b2, W3, b3, W4, b4 = conv_split_params(params, r)
    x = np.asarray(x, np.float64)
    n, pix = x.shape[0], r * r
    X1 = im2col(x[:, :pix].reshape(n, r, r, 1), r)
    z1 = rb(X1) @ rb(W1) + b1
    a1 = np.maximum(z1, 0)
    X2 = im2col(a1.reshape(n, r, r, CONV_C1), r)
    z2 = rb(X2) @ rb(W2) + b2
    a2 = np.maximum(z2, 0)
    H = np.concatenate([a2.reshape(n, pix * CONV_C2), x[:, pix:pix + 2]], axis=1)
    z3 = rb(H) @ rb(W3) + b3
    a3 = np.maximum(z3, 0)
    y = rb(a3) @ rb(W4) + b4
    return y, (X1, z1, X2, z2, H, z3, a3)


def _loss_dy(y, t, valid, classes):
    """Masked weighted MSE (+ count cross-entropy) over the batch and dL/dy."""
    n, nu = y.shape[0], t.shape[1]
    e = y[:, :nu] - t
    tw = TARGET_WEIGHT_2E if nu == 8 else TARGET_WEIGHT[:nu]
    loss = float(np.sum(tw * e * e * valid[:, None]) / n)
    dy = np.zeros_like(y)
    dy[:, :nu] = 2.0 * tw * e * valid[:, None] / n
    if classes is not None:
        c = np.asarray(classes).astype(np.int64)
        lab = c >= 0
        lg = y[:, COUNT0:COUNT0 + CLASSES]
        p = np.exp(lg - lg.max(axis=1, keepdims=True))
        p /= p.sum(axis=1, keepdims=True)
        rows = np.nonzero(lab)[0]
        loss += float(COUNT_WEIGHT * np.sum(-np.log(p[rows, c[rows]])) / n)
        onehot = np.zeros_like(p)
        onehot[rows, c[rows]] = 1.0
        dy[:, COUNT0:COUNT0 + CLASSES] = COUNT_WEIGHT * (p - onehot) * lab[:, None] / n
    return loss, dy


def conv_loss_and_grad(params, x, t, valid, r, classes=None, exact=False):
    """Loss and parameter gradient of the conv net, with the GPU's bfloat16
    rounding of every GEMM operand of the backward pass unless exact."""
    rb = (lambda a: np.asarray(a, np.float64)) if exact else bf16
    W1, b1, W2, b2, W3, b3, W4, b4 = conv_split_params(params, r)
    y, (X1, z1, X2, z2, H, z3, a3) = conv_forward(params, x, r, exact)
    n, pix = y.shape[0], r * r
    loss, dy = _loss_dy(y, np.asarray(t, np.float64), np.asarray(valid, np.float64), classes)
    gW4 = rb(a3).T @ rb(dy)
    gb4 = dy.sum(axis=0)
    d3 = (rb(dy) @ rb(W4).T) * (z3 > 0)
    gW3 = rb(H).T @ rb(d3)
    gb3 = d3.sum(axis=0)
    d2 = (rb(d3) @ rb(W3[:pix * CONV_C2]).T).reshape(n * pix, CONV_C2) * (z2 > 0)
    gW2 = rb(X2).T @ rb(d2)
    gb2 = d2.sum(axis=0)
    d1 = col2im(rb(d2) @ rb(W2).T, n, r, CONV_C1) * (z1 > 0)
    gW1 = rb(X1).T @ rb(d1)
    gb1 = d1.sum(axis=0)
    grad = np.concatenate([g.ravel() for g in (gW1, gb1, gW2, gb2, gW3, gb3, gW4, gb4)])
    return loss, grad, y


def conv_init(r, seed):
    """He-style uniform initial parameters (a test helper; the library draws its own)."""
    rng = np.random.default_rng(seed)
    parts = []
    for fan_in, shape in ((9, (9, CONV_C1)), (None, (CONV_C1,)), (9 * CONV_C1, (9 * CONV_C1, CONV_C2)),
                          (None, (CONV_C2,)), (r * r * CONV_C2 + 2, (r * r * CONV_C2 + 2, CONV_FC)),
                          (None, (CONV_FC,)), (CONV_FC, (CONV_FC, N_OUT)), (None, (N_OUT,))):
        if fan_in is None:
            parts.append(np.zeros(shape))
        else:
            parts.append(rng.uniform(-1, 1, shape) * np.sqrt(6.0 / fan_in))
    return np.concatenate([a.ravel() for a in parts])
