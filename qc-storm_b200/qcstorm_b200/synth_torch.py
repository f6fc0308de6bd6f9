"""The workloads of synth.py drawn with torch, so that millions of ROI records
are made where they are used (on the GPU) instead of on the host.

Same distributions, record layout and parameters as synth.gs2d_rois,
synth.as3d_rois and synth.multi_rois (expected counts at pixel centres,
Poisson noise, header words [x, y, frame % 65536, frame // 65536, type] with
the ROI centred at (1024, 1024), one ROI per frame); a different random
stream, so the records are not those of the numpy generators.  Records are
returned as an int16 tensor holding the uint16 bit patterns (the C ABI reads
them as uint16), truth as float64 tensors on the same device.
"""
import math

import torch

from . import synth

KINDS = ("gs2d", "as3d", "multi")


def _u(g, n, a, b, dev):
    return torch.rand(n, generator=g, device=dev, dtype=torch.float64) * (b - a) + a


def _log_u(g, n, a, b, dev):
    return torch.exp(_u(g, n, math.log(a), math.log(b), dev))


def _gauss(R, x0, y0, sx, sy, amp):
    c = torch.arange(R, device=x0.device, dtype=torch.float64) + 0.5
    gx = torch.exp(-((c[None, :] - x0[:, None]) ** 2) / (2 * sx[:, None] ** 2))
    gy = torch.exp(-((c[None, :] - y0[:, None]) ** 2) / (2 * sy[:, None] ** 2))
    return amp[:, None, None] * gy[:, :, None] * gx[:, None, :]


def _records(counts, first_frame):
    n, R, _ = counts.shape
    rec = torch.zeros((n, R * (R + 1)), dtype=torch.int32, device=counts.device)
    rec[:, :R * R] = counts.reshape(n, R * R).to(torch.int32)
    rec[:, R * R + 0] = 1024
    rec[:, R * R + 1] = 1024
    fr = first_frame + torch.arange(n, device=counts.device, dtype=torch.int64)
    rec[:, R * R + 2] = (fr % 65536).to(torch.int32)
    rec[:, R * R + 3] = (fr // 65536).to(torch.int32)
    # uint16 bit patterns in int16 storage
    return torch.where(rec > 32767, rec - 65536, rec).to(torch.int16)


def para(kind, R):
    """The localization parameters of a workload (those of the numpy generator)."""
    if kind == "gs2d":
        return synth.gs2d_rois(1, R=R)[1]
    if kind == "as3d":
        return synth.as3d_rois(1, R=R)[1]
    return synth.multi_rois(1, R=R)[1]


def rois(kind, n, R, seed, device="cuda", first_frame=1):
    """(records [n, R*(R+1)] int16, truth dict of float64 tensors) of workload
    `kind` ("gs2d", "as3d" or "multi"); records of frames first_frame ..
    first_frame + n - 1."""
    dev = torch.device(device)
    g = torch.Generator(device=dev)
    g.manual_seed(int(seed))
    if kind == "gs2d":
        sig = _u(g, n, 1.0, 1.6, dev)
        x0 = R / 2 + _u(g, n, -0.5, 0.5, dev)
        y0 = R / 2 + _u(g, n, -0.5, 0.5, dev)
        ph = _log_u(g, n, 500, 5000, dev)
        bg = _u(g, n, 20, 100, dev)
        mu = _gauss(R, x0, y0, sig, sig, ph / (2 * math.pi * sig ** 2)) + bg[:, None, None]
        counts = torch.clamp(torch.poisson(mu, generator=g), max=65535)
        truth = dict(x=x0, y=y0, sigma=sig, photons=ph, background=bg)
    elif kind == "as3d":
        s0, c, d = synth.AS3D_S0, synth.AS3D_C, synth.AS3D_D
        z = _u(g, n, -600, 600, dev)
        sx = s0 * torch.sqrt(1 + ((z - c) / d) ** 2)
        sy = s0 * torch.sqrt(1 + ((z + c) / d) ** 2)
        x0 = R / 2 + _u(g, n, -0.5, 0.5, dev)
        y0 = R / 2 + _u(g, n, -0.5, 0.5, dev)
        ph = _log_u(g, n, 1000, 8000, dev)
        bg = _u(g, n, 20, 150, dev)
        mu = _gauss(R, x0, y0, sx, sy, ph / (2 * math.pi * sx * sy)) + bg[:, None, None]
        e = torch.poisson(mu, generator=g)
        counts = torch.clamp(torch.round(e / 0.45 + 100), 0, 65535)
        truth = dict(x=x0, y=y0, z=z, sigma_x=sx, sigma_y=sy, photons=ph, background=bg)
    elif kind == "multi":
        r = _u(g, n, 0, 1, dev)
        k = 1 + (r >= 0.5).to(torch.int64) + (r >= 0.8).to(torch.int64)
        sig = _u(g, n, 1.0, 1.5, dev)
        bg = _u(g, n, 20, 100, dev)
        xs = torch.full((n, 3), float("nan"), dtype=torch.float64, device=dev)
        ys = torch.full((n, 3), float("nan"), dtype=torch.float64, device=dev)
        xs[:, 0] = R / 2 + _u(g, n, -0.5, 0.5, dev)
        ys[:, 0] = R / 2 + _u(g, n, -0.5, 0.5, dev)
        ang = _u(g, n, 0, 2 * math.pi, dev)
        for j in (1, 2):
            sep = _u(g, n, 1, 3, dev)
            a = ang + (j - 1) * _u(g, n, math.pi / 3, 5 * math.pi / 3, dev)
            xs[:, j] = xs[:, 0] + sep * torch.cos(a)
            ys[:, j] = ys[:, 0] + sep * torch.sin(a)
        ph = torch.stack([_log_u(g, n, 500, 5000, dev) for _ in range(3)], 1)
        mu = bg[:, None, None].expand(n, R, R).clone()
        for j in range(3):
            on = k > j
            amp = torch.where(on, ph[:, j] / (2 * math.pi * sig ** 2), torch.zeros_like(sig))
            mu += _gauss(R, torch.where(on, xs[:, j], 0.0), torch.where(on, ys[:, j], 0.0), sig, sig, amp)
        counts = torch.clamp(torch.poisson(mu, generator=g), max=65535)
        off = k[:, None] <= torch.arange(3, device=dev)[None, :]
        xs[off] = float("nan")
        ys[off] = float("nan")
        truth = dict(k=k, x=xs, y=ys, sigma=sig, photons=torch.where(off, torch.zeros_like(ph), ph), background=bg)
    else:
        raise ValueError("unknown workload %r" % (kind,))
    return _records(counts, first_frame), truth
