"""Seeded localization rows for the render tests: positions over the whole
super-resolution image (borders included), SNR around the threshold, CRLB
widths from 2 to 40 nm with NaN, zero and negative entries, z inside and
outside the depth range, clusters so that splats overlap."""
import numpy as np

from qcstorm_b200.abi import default_para


def render_para(loc_type=0, width=64, high=48, zoom=5.0):
    p = default_para(LocType=loc_type, ROISize=7)
    p.ImageWidth, p.ImageHigh, p.PixelZoom, p.PixelSize = width, high, zoom, 100.0
    p.SRImageWidth = (int(width * zoom) + 3) // 4 * 4
    p.SRImageHigh = (int(high * zoom) + 3) // 4 * 4
    p.SNR_th = 5.0
    p.MinZDepth, p.MaxZDepth = -500.0, 500.0
    return p


def render_rows(n, para, seed):
    rng = np.random.default_rng(seed)
    rows = np.zeros((n, 12), np.float32)
    centres = rng.uniform(0, [para.ImageWidth, para.ImageHigh], size=(max(n // 20, 1), 2))
    pick = rng.integers(0, centres.shape[0], n)
    xy = centres[pick] + rng.normal(0, 0.6, (n, 2))
    edge = rng.random(n) < 0.1
    xy[edge] = rng.uniform(-1, [para.ImageWidth + 1, para.ImageHigh + 1], size=(edge.sum(), 2))
    rows[:, 0] = np.exp(rng.uniform(np.log(0.5), np.log(3000), n))
    rows[:, 1:3] = xy
    rows[:, 3] = rng.uniform(-3000, 3000, n) * (rng.random(n) < 0.1) + rng.uniform(-600, 600, n)
    rows[:, 8] = rng.uniform(2, 40, n)
    crlb = rng.uniform(2, 40, (n, 2))
    bad = rng.random(n)
    crlb[bad < 0.02, 0] = np.nan
    crlb[(bad >= 0.02) & (bad < 0.04), 0] = 0
    crlb[(bad >= 0.04) & (bad < 0.05), 0] = -3
    rows[:, 9:11] = crlb
    rows[:, 11] = rng.integers(1, 100, n)
    return rows
