"""The FP64 Fisher-matrix CRLB oracle (oracle/qcs_oracle_fisher.c), on the
CPU: closed forms, and the reference's own diagonal CRLB where the two
bounds coincide.

The reference's CRLB columns (LocPrecCalc_GaussianCRLB.h:65-243) are the
Fisher information of x alone, from numerical second derivatives (step 0.02)
on a fixed 9x9 grid with the emitter at the grid centre and read noise added
to the background.  For an emitter at the centre of a 9x9 ROI the full bound
of x decouples from photons, background and width (their derivatives are
even in x, its own is odd), so the oracle's x bound must equal the
reference's column 9 up to the numerical derivative's error.
"""
import numpy as np
import pytest

import oracle_lib as O
from qcstorm_b200 import abi


def rows_gs2d(total, bkg, sigma, n=1):
    r = np.zeros((n, 12), np.float32)
    r[:, 0] = total / (2 * np.pi * sigma ** 2)
    r[:, 4] = sigma
    r[:, 5] = sigma
    r[:, 6] = total
    r[:, 7] = bkg
    return r


def test_high_photon_limit_is_sigma_over_sqrt_n():
    # no background, no read noise, pixels much finer than the PSF in effect:
    # CRLB_x = sigma / sqrt(N) (the classical bound without pixelation)
    p = abi.default_para(ROISize=17, LocType=0, QE=1.0, ReadNoise_e=0.0, PixelSize=100.0)
    for sigma in (1.2, 1.6):
        r = rows_gs2d(1e6, 1e-6, sigma)
        o = O.crlb_fisher(p, r)
        assert o[0, 7] == 0
        assert o[0, 0] == pytest.approx(100.0 * sigma / 1e3, rel=2e-3)
        assert o[0, 1] == pytest.approx(o[0, 0], rel=1e-6)
        assert o[0, 3] == pytest.approx(1e3, rel=1e-2)  # Poisson: sqrt(N) photons


def test_scaling_and_invalid_rows():
    p = abi.default_para(ROISize=7, LocType=0, QE=0.72, ReadNoise_e=1.3, PixelSize=100.0)
    r = np.concatenate([rows_gs2d(2000, 50, 1.3), rows_gs2d(8000, 50, 1.3), rows_gs2d(2000, 50, 1.3)])
    r[2, 0] = 0  # a rejected (zero) row
    o = O.crlb_fisher(p, r)
    assert list(o[:, 7]) == [0, 0, 1]
    assert o[1, 0] < o[0, 0] / 1.5  # four times the photons: a smaller bound
    assert np.all(o[2, :7] == 0)


def centred_rows(n, seed):
    rng = np.random.default_rng(seed)
    total = np.exp(rng.uniform(np.log(500), np.log(5000), n))
    bkg = rng.uniform(20, 100, n)
    sig = rng.uniform(1.0, 1.6, n)
    return np.concatenate([rows_gs2d(t, b, s) for t, b, s in zip(total, bkg, sig)])


def reference_diagonal_f64(row, rn2, h=0.02):
    """The reference's diagonal estimate of x (LocPrecCalc_GaussianCRLB.h:
    130-243: model on the 9x9 grid of offsets -4..4 around the emitter,
    background + read noise^2, FI = sum d2(mu) - mu d2(log mu) by central
    second differences with step h) evaluated in double."""
    t, b, s = float(row[6]), float(row[7]), float(row[4])
    c = np.arange(9) - 4.0
    X, Y = np.meshgrid(c, c)

    def mu(x0):
        return t / (2 * np.pi * s * s) * np.exp(-((X - x0) ** 2 + Y ** 2) / (2 * s * s)) + b + rn2

    m0, mp, mn = mu(0.0), mu(h), mu(-h)
    d2 = (mp - 2 * m0 + mn) / h / h
    d2l = (np.log(mp) - 2 * np.log(m0) + np.log(mn)) / h / h
    return 1.0 / np.sqrt(np.sum(d2 - m0 * d2l))


def test_centred_x_bound_equals_reference_formula_in_double():
    r = centred_rows(300, 3)
    p = abi.default_para(ROISize=9, LocType=0, QE=1.0, ReadNoise_e=1.3, PixelSize=100.0)
    o = O.crlb_fisher(p, r)
    assert np.all(o[:, 7] == 0)
    want = np.array([reference_diagonal_f64(x, 1.3 ** 2) for x in r]) * 100.0
    np.testing.assert_allclose(o[:, 0], want, rtol=1e-4)  # the second difference's own error
    np.testing.assert_allclose(o[:, 1], want, rtol=1e-4)


def test_centred_x_bound_against_reference_host_build():
    # the reference's float32 second difference of log(mu) with step 0.02
    # carries ~1e-3 absolute error per pixel: its estimate scatters around
    # the exact bound (median 0.1%, 95th percentile 1.4% on these rows)
    if O.ref_host() is None:
        pytest.skip("reference host build not present")
    r = centred_rows(2000, 3)
    p = abi.default_para(ROISize=9, LocType=0, QE=1.0, ReadNoise_e=1.3, PixelSize=100.0)
    o = O.crlb_fisher(p, r)
    diag = O.crlb(p, r, lib="ref")
    rel = o[:, 0] / diag[:, 9] - 1
    assert np.median(np.abs(rel)) < 0.005
    assert abs(rel.mean()) < 0.003
    assert np.percentile(np.abs(rel), 95) < 0.03


def test_as3d_z_bound_is_the_jacobian_of_the_calibration():
    from qcstorm_b200 import synth
    cal = synth.as3d_calibration()
    p = abi.default_para(ROISize=9, LocType=1, QE=1.0, ReadNoise_e=1.3, PixelSize=100.0, **cal)
    r = np.zeros((2, 12), np.float32)
    r[:, 6] = 4000
    r[:, 7] = 60
    r[:, 0] = 1
    r[0, 4], r[0, 5] = 1.2, 1.6
    r[1, 4], r[1, 5] = 1.6, 1.2
    o = O.crlb_fisher(p, r)
    assert np.all(o[:, 7] == 0)
    # mirrored widths: same x / y bounds swapped, same z bound (linear calibration)
    assert o[0, 0] == pytest.approx(o[1, 1], rel=1e-6)
    assert o[0, 5] == pytest.approx(o[1, 6], rel=1e-6)
    assert o[0, 2] == pytest.approx(o[1, 2], rel=1e-6)
    # z = p1 (sx^2 - sy^2): its bound is at least |dz/dsx| * CRLB(sx) when sy is known exactly
    p1 = cal["p1_XGY"]
    assert o[0, 2] >= 0.5 * abs(2 * p1 * 1.2) * o[0, 5]
