"""Seeded synthetic single-molecule data in the reference's record formats.

Each generator returns ROI records (N x R*(R+1) uint16, pixels then header
words [x, y, frame%65536, frame//65536, detector type]), the localization
parameters that describe the camera, and the ground truth.  Expected counts
are sampled at pixel centres, the reference's model convention
(bfgsMLE_GS2D_core.h:495-501: pixel (row, col) centred at (col+0.5, row+0.5)).

Workloads (sizes are the callers'):
  gs2d_rois       symmetric Gaussian, sigma ~ U(1.0, 1.6) px, centre = ROI centre
                  + U(-0.5, 0.5), photons log-U[500, 5000], background U(20, 100)
                  e-/px, Poisson; stored as e- counts (Offset 0, KAdc 1, QE 1).
  as3d_rois       astigmatic, z ~ U(-600, 600) nm, sigma_x = s0*sqrt(1+((z-c)/d)^2),
                  sigma_y = s0*sqrt(1+((z+c)/d)^2), s0 = 1.3 px, c = 250 nm,
                  d = 400 nm; photons log-U[1000, 8000], background U(20, 150);
                  ADU = round(e-/0.45 + 100).
  multi_rois      1/2/3 emitters w.p. 0.5/0.3/0.2, separation U(1, 3) px, shared
                  sigma ~ U(1.0, 1.5) and background U(20, 100), per-emitter
                  photons log-U[500, 5000]; e- counts.
  frames          full frames: Poisson(density) emitters per frame, uniform in the
                  field of view with a fraction placed in close pairs (< 3 px).
"""
import numpy as np

from .abi import default_para


def _records(img, frames, xy=None, det=None):
    n, R, _ = img.shape
    rec = np.zeros((n, R * (R + 1)), np.uint16)
    rec[:, :R * R] = img.reshape(n, R * R)
    if xy is None:
        rec[:, R * R + 0] = 1024
        rec[:, R * R + 1] = 1024
    else:
        rec[:, R * R + 0] = xy[:, 0]
        rec[:, R * R + 1] = xy[:, 1]
    frames = np.asarray(frames, np.int64)
    rec[:, R * R + 2] = (frames % 65536).astype(np.uint16)
    rec[:, R * R + 3] = (frames // 65536).astype(np.uint16)
    if det is not None:
        rec[:, R * R + 4] = det
    return rec


def _gauss(R, x0, y0, sx, sy, amp):
    c = np.arange(R, dtype=np.float64) + 0.5
    gx = np.exp(-((c[None, :] - x0[:, None]) ** 2) / (2 * sx[:, None] ** 2))
    gy = np.exp(-((c[None, :] - y0[:, None]) ** 2) / (2 * sy[:, None] ** 2))
    return amp[:, None, None] * gy[:, :, None] * gx[:, None, :]


def gs2d_rois(n, R=7, seed=0, first_frame=1):
    """Symmetric 2D single-emitter ROIs (one ROI per frame, isolated)."""
    rng = np.random.default_rng(seed)
    sig = rng.uniform(1.0, 1.6, n)
    x0 = R / 2 + rng.uniform(-0.5, 0.5, n)
    y0 = R / 2 + rng.uniform(-0.5, 0.5, n)
    ph = np.exp(rng.uniform(np.log(500), np.log(5000), n))
    bg = rng.uniform(20, 100, n)
    mu = _gauss(R, x0, y0, sig, sig, ph / (2 * np.pi * sig ** 2)) + bg[:, None, None]
    img = np.minimum(rng.poisson(mu), 65535).astype(np.uint16)
    rec = _records(img, first_frame + np.arange(n))
    para = default_para(Offset=0.0, KAdc=1.0, QE=1.0, ROISize=R, LocType=0, MultiEmitterFitEn=0)
    truth = dict(x=x0, y=y0, sigma=sig, photons=ph, background=bg)
    return rec, para, truth


AS3D_S0, AS3D_C, AS3D_D = 1.3, 250.0, 400.0


def as3d_calibration():
    """z(sigma_x^2 - sigma_y^2) of the generator: sigma_x^2 - sigma_y^2 =
    -4 z c s0^2 / d^2, so both sign branches are the linear term
    p1 = -d^2 / (4 c s0^2) nm/px^2 (p4..p2 = p0 = 0)."""
    p1 = -(AS3D_D ** 2) / (4 * AS3D_C * AS3D_S0 ** 2)
    return dict(p4_XGY=0.0, p3_XGY=0.0, p2_XGY=0.0, p1_XGY=p1, p0_XGY=0.0,
                p4_XLY=0.0, p3_XLY=0.0, p2_XLY=0.0, p1_XLY=p1, p0_XLY=0.0)


def as3d_rois(n, R=9, seed=0, first_frame=1):
    """Astigmatic 3D single-emitter ROIs in camera ADU (offset 100, 0.45 e-/ADU)."""
    rng = np.random.default_rng(seed)
    z = rng.uniform(-600, 600, n)
    sx = AS3D_S0 * np.sqrt(1 + ((z - AS3D_C) / AS3D_D) ** 2)
    sy = AS3D_S0 * np.sqrt(1 + ((z + AS3D_C) / AS3D_D) ** 2)
    x0 = R / 2 + rng.uniform(-0.5, 0.5, n)
    y0 = R / 2 + rng.uniform(-0.5, 0.5, n)
    ph = np.exp(rng.uniform(np.log(1000), np.log(8000), n))
    bg = rng.uniform(20, 150, n)
    mu = _gauss(R, x0, y0, sx, sy, ph / (2 * np.pi * sx * sy)) + bg[:, None, None]
    e = rng.poisson(mu)
    adu = np.clip(np.rint(e / 0.45 + 100), 0, 65535).astype(np.uint16)
    rec = _records(adu, first_frame + np.arange(n))
    para = default_para(Offset=100.0, KAdc=0.45, QE=1.0, ROISize=R, LocType=1, MultiEmitterFitEn=0,
                        **as3d_calibration())
    truth = dict(x=x0, y=y0, z=z, sigma_x=sx, sigma_y=sy, photons=ph, background=bg)
    return rec, para, truth


def multi_rois(n, R=11, seed=0, first_frame=1):
    """Multi-emitter 2D ROIs with 1..3 emitters."""
    rng = np.random.default_rng(seed)
    k = rng.choice([1, 2, 3], size=n, p=[0.5, 0.3, 0.2])
    sig = rng.uniform(1.0, 1.5, n)
    bg = rng.uniform(20, 100, n)
    xs = np.full((n, 3), np.nan)
    ys = np.full((n, 3), np.nan)
    ph = np.zeros((n, 3))
    xs[:, 0] = R / 2 + rng.uniform(-0.5, 0.5, n)
    ys[:, 0] = R / 2 + rng.uniform(-0.5, 0.5, n)
    ang = rng.uniform(0, 2 * np.pi, n)
    for j in (1, 2):
        sep = rng.uniform(1, 3, n)
        a = ang + (j - 1) * rng.uniform(np.pi / 3, 5 * np.pi / 3, n)
        xs[:, j] = xs[:, 0] + sep * np.cos(a)
        ys[:, j] = ys[:, 0] + sep * np.sin(a)
    for j in range(3):
        ph[:, j] = np.exp(rng.uniform(np.log(500), np.log(5000), n))
    mu = np.repeat(bg[:, None, None], R, 1).repeat(R, 2).astype(np.float64)
    for j in range(3):
        on = k > j
        amp = np.where(on, ph[:, j] / (2 * np.pi * sig ** 2), 0.0)
        xx = np.where(on, xs[:, j], 0.0)
        yy = np.where(on, ys[:, j], 0.0)
        mu += _gauss(R, xx, yy, sig, sig, amp)
    img = np.minimum(rng.poisson(mu), 65535).astype(np.uint16)
    rec = _records(img, first_frame + np.arange(n))
    para = default_para(Offset=0.0, KAdc=1.0, QE=1.0, ROISize=R, LocType=0, MultiEmitterFitEn=1)
    for j in range(3):
        xs[k <= j, j] = np.nan
        ys[k <= j, j] = np.nan
    truth = dict(k=k, x=xs, y=ys, sigma=sig, photons=np.where(k[:, None] > np.arange(3), ph, 0), background=bg)
    return rec, para, truth


def frames(n_frames, width=2048, height=2048, density=3000, pair_frac=0.2, seed=0, offset=100.0,
           kadc=0.45, sigma=(1.0, 1.6), photons=(500, 5000), background=(20, 100)):
    """Full camera frames (n_frames x height x width uint16 ADU) and their emitters.

    Emitters: Poisson(density) per frame, uniform in the field of view; a
    fraction pair_frac of them gets a partner < 3 px away.  PSF, photons and
    background are drawn as for gs2d_rois; ADU = round(e-/kadc + offset).
    """
    rng = np.random.default_rng(seed)
    out = np.empty((n_frames, height, width), np.uint16)
    truth = []
    half = 7
    for f in range(n_frames):
        m = rng.poisson(density)
        npair = int(round(m * pair_frac / 2))
        nsingle = m - 2 * npair
        x = rng.uniform(8, width - 8, nsingle + npair)
        y = rng.uniform(8, height - 8, nsingle + npair)
        a = rng.uniform(0, 2 * np.pi, npair)
        d = rng.uniform(1, 3, npair)
        x = np.concatenate([x, x[nsingle:] + d * np.cos(a)])
        y = np.concatenate([y, y[nsingle:] + d * np.sin(a)])
        cnt = x.size
        sig = rng.uniform(sigma[0], sigma[1], cnt)
        ph = np.exp(rng.uniform(np.log(photons[0]), np.log(photons[1]), cnt))
        bgv = rng.uniform(background[0], background[1])
        mu = np.full((height, width), bgv, np.float64)
        ix = np.floor(x).astype(int)
        iy = np.floor(y).astype(int)
        offs = np.arange(-half, half + 1)
        for j in range(cnt):
            xs = np.clip(ix[j] + offs, 0, width - 1)
            ys = np.clip(iy[j] + offs, 0, height - 1)
            gx = np.exp(-((xs + 0.5 - x[j]) ** 2) / (2 * sig[j] ** 2))
            gy = np.exp(-((ys + 0.5 - y[j]) ** 2) / (2 * sig[j] ** 2))
            mu[np.ix_(ys, xs)] += ph[j] / (2 * np.pi * sig[j] ** 2) * np.outer(gy, gx)
        e = rng.poisson(mu)
        out[f] = np.clip(np.rint(e / kadc + offset), 0, 65535).astype(np.uint16)
        truth.append(dict(x=x, y=y, sigma=sig, photons=ph, background=bgv))
    para = default_para(Offset=offset, KAdc=kadc, QE=1.0, ImageWidth=width, ImageHigh=height)
    return out, para, truth


def blinking_rows(n_emitters=400, frames=12, seed=0, width=256, jitter=0.1, loc_type=0, first_frame=1):
    """Rows (12 floats) of emitters that switch on and off (on -> on 0.6,
    off -> on 0.25) over `frames` frames; each on-frame gives one row near the
    emitter's position (Gaussian jitter in px).  Returns (rows, per-frame counts)."""
    rng = np.random.default_rng(seed)
    ex = rng.uniform(5, width - 5, n_emitters)
    ey = rng.uniform(5, width - 5, n_emitters)
    ez = rng.uniform(-400, 400, n_emitters)
    on = rng.random(n_emitters) < 0.4
    rows, counts = [], []
    for f in range(frames):
        if f:
            stay = rng.random(n_emitters) < 0.6
            come = rng.random(n_emitters) < 0.25
            on = np.where(on, stay, come)
        idx = np.nonzero(on)[0]
        rng.shuffle(idx)
        k = idx.size
        r = np.zeros((k, 12), np.float32)
        sig = rng.uniform(1.0, 1.5, k)
        peak = np.exp(rng.uniform(np.log(200), np.log(2000), k))
        bkg = rng.uniform(20, 80, k)
        r[:, 0] = peak
        r[:, 1] = ex[idx] + rng.normal(0, jitter, k)
        r[:, 2] = ey[idx] + rng.normal(0, jitter, k)
        r[:, 3] = ez[idx] + rng.normal(0, 20, k) if loc_type == 1 else 0.0
        r[:, 4] = sig
        r[:, 5] = sig * (rng.uniform(0.8, 1.25, k) if loc_type == 1 else 1.0)
        r[:, 6] = peak * 2 * np.pi * r[:, 4] * r[:, 5]
        r[:, 7] = bkg
        r[:, 8] = peak / np.sqrt(peak + bkg)
        r[:, 9] = rng.uniform(5, 30, k)
        r[:, 10] = rng.uniform(5, 30, k)
        r[:, 11] = first_frame + f
        rows.append(r)
        counts.append(k)
    return np.concatenate(rows), np.array(counts)


def group_sizes(counts, frames_per_group):
    """Rows per group of `frames_per_group` consecutive frames."""
    return np.array([counts[i:i + frames_per_group].sum() for i in range(0, counts.size, frames_per_group)],
                    np.int32)
