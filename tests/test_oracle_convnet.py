"""The conv start-point network's numpy restatement (oracle/qcs_net_oracle.py)
checked against itself: the analytic gradient of conv_loss_and_grad (exact
mode, no bfloat16 rounding) against central finite differences of the loss,
and im2col / col2im as adjoint maps.  The GPU training kernels are then
checked against this gradient in tests/test_gpu_convnet.py."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import qcs_net_oracle as NO  # noqa: E402


def test_im2col_col2im_adjoint():
    rng = np.random.default_rng(1)
    n, r, c = 3, 5, 4
    a = rng.normal(size=(n, r, r, c))
    d = rng.normal(size=(n * r * r, 9 * c))
    lhs = np.sum(NO.im2col(a, r) * d)
    rhs = np.sum(a.reshape(n * r * r, c) * NO.col2im(d, n, r, c))
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs)


def test_im2col_taps():
    """Tap t = 3 (dy + 1) + (dx + 1) reads the pixel at (y + dy, x + dx)."""
    r = 4
    a = np.arange(r * r, dtype=np.float64).reshape(1, r, r, 1) + 1
    cols = NO.im2col(a, r).reshape(r, r, 9)
    assert cols[1, 2, 0] == a[0, 0, 1, 0]  # dy = -1, dx = -1
    assert cols[1, 2, 8] == a[0, 2, 3, 0]  # dy = +1, dx = +1
    assert cols[0, 0, 0] == 0.0 and cols[3, 3, 8] == 0.0


def test_conv_gradient_finite_differences():
    r = 5
    rng = np.random.default_rng(2)
    n = 6
    x = np.zeros((n, NO.in_width(r)))
    x[:, :r * r] = rng.uniform(0, 1, (n, r * r))
    x[:, r * r] = 0.5
    x[:, r * r + 1] = 0.3
    p = NO.conv_init(r, 3)
    p += rng.normal(scale=0.01, size=p.size)  # non-zero biases
    t = rng.normal(size=(n, 5))
    v = np.array([1, 1, 0, 1, 1, 1], np.float64)
    cls = np.array([0, 1, 2, -1, 1, 0])
    loss, g, _ = NO.conv_loss_and_grad(p, x, t, v, r, classes=cls, exact=True)
    assert g.size == NO.conv_param_count(r)
    idx = rng.choice(p.size, 60, replace=False)
    # every parameter block at least once
    bounds = np.cumsum([9 * 32, 32, 288 * 64, 64, (r * r * 64 + 2) * 256, 256, 256 * 8, 8])
    idx = np.concatenate([idx, bounds - 1, bounds[:-1]])
    h = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        lp = NO.conv_loss_and_grad(pp, x, t, v, r, classes=cls, exact=True)[0]
        lm = NO.conv_loss_and_grad(pm, x, t, v, r, classes=cls, exact=True)[0]
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(fd)), (i, fd, g[i])
