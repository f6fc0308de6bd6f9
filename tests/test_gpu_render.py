"""Super-resolution render on the GPU (qcs_render_*).

The kernel adds each row's 7x7 Gaussian with float atomics, so the order of
the additions differs from the oracle's row order (and between runs, as in
the reference); the images are compared within that rounding and the
difference of __expf from glibc expf (relative 1e-4, absolute 1e-3 photons).
The row selection, the weights and the widths are the reference's: checked
against the render oracle (pinned bit for bit to the reference's host build)
and against the reference's own render kernels built for sm_100a, for every
mode, 2D and 3D.  The display maximum and histogram read the image while
other rows are still being added (in the reference too), so they are compared
in range.  The device hand-off renders a localization's rows with their count
read on the device and gives the host path's image.
"""
import numpy as np
import pytest

import oracle_lib as O
from qcstorm_b200 import lib as qlib
from qcstorm_b200 import synth
from render_rows import render_para, render_rows

pytestmark = pytest.mark.gpu


def close(a, b):
    np.testing.assert_allclose(a, b, rtol=1e-4, atol=1e-3)


@pytest.mark.parametrize("loc_type,mode", [(0, 0), (0, 1), (0, 2), (0, 3), (1, 0), (1, 1), (1, 2), (2, 0)])
def test_render_matches_oracle_and_reference(cuda_ok, loc_type, mode):
    p = render_para(loc_type)
    rows = render_rows(4000, p, seed=3 + mode + 10 * loc_type)
    r = qlib.RenderContext(p, capacity=4000)
    r.render(rows, mode, fixed_prec=12.5)
    img, cmap, mx, hist = r.read()
    r.close()
    o_img, o_cmap, o_max, o_hist = O.render(p, rows, mode, fixed_prec=12.5)
    assert o_img.sum() > 0
    close(img, o_img)
    if loc_type != 0:
        np.testing.assert_allclose(cmap, o_cmap, rtol=1e-4, atol=0.5)  # z (nm) times the weights
    # the running maximum: from centres read mid-way, bounded by the final image's centres
    assert 0 < mx <= int(o_img.max()) + 1
    # histogram: a row whose centre is the running maximum at its moment, or
    # which sees the maximum still at 0, is not binned; which rows those are
    # depends on the order the rows run in
    assert 0 < hist.sum() <= o_img.size and 0 < o_hist.sum()
    assert hist.sum() <= rows.shape[0]
    g_img, g_cmap, _, _ = O.render(p, rows, mode, fixed_prec=12.5, lib="ref_gpu")
    close(img, g_img)
    if loc_type != 0:
        np.testing.assert_allclose(cmap, g_cmap, rtol=1e-4, atol=0.5)


def test_render_accumulates_and_resets(cuda_ok):
    p = render_para(0)
    a, b = render_rows(2000, p, seed=1), render_rows(2000, p, seed=2)
    r = qlib.RenderContext(p, capacity=2000)
    r.render(a)
    r.render(b)
    img = r.read()[0]
    close(img, O.render(p, b, 0, state=O.render(p, a, 0))[0])
    r.reset(display=False)
    img2, _, mx2, hist2 = r.read()
    assert not img2.any() and mx2 > 0 and hist2.sum() > 0
    r.reset()
    _, _, mx3, hist3 = r.read()
    assert mx3 == 0 and not hist3.any()
    r.close()


def test_render_refuses_mismatch(cuda_ok):
    p = render_para(0)
    r = qlib.RenderContext(p, capacity=100)
    with pytest.raises(RuntimeError):
        r.render(render_rows(101, p, seed=1))
    q = render_para(0, width=80)
    with pytest.raises(RuntimeError):
        r.render(render_rows(10, q, seed=1), para=q)
    with pytest.raises(RuntimeError):
        r.render(render_rows(10, p, seed=1), mode=7)
    r.close()


def test_render_hand_off_from_localization(cuda_ok):
    """Frames -> extraction -> localization -> render, the rows and their count
    never leaving the device; the image equals the render of the same rows
    read back to the host."""
    import torch
    fr, para, _ = synth.frames(6, width=256, height=256, density=150, seed=17)
    para.MultiEmitterFitEn = 1
    para.PixelZoom = 4.0
    para.SRImageWidth = (int(para.ImageWidth * para.PixelZoom) + 3) // 4 * 4
    para.SRImageHigh = (int(para.ImageHigh * para.PixelZoom) + 3) // 4 * 4
    ex = qlib.ExtractContext(para, max_batched_num=1, capacity=20000)
    loc = qlib.LocContext(para, capacity=20000)
    s = torch.cuda.Stream()
    sh = s.cuda_stream
    d_fr = torch.from_numpy(fr.view(np.int16)).cuda()
    fb = para.ImageWidth * para.ImageHigh * 2
    for f in range(fr.shape[0]):
        ex.extract_device(d_fr.data_ptr() + f * fb, 1, f, stream=sh)
    d_rois, d_wle, d_n = ex.device_records()
    loc.localize_device_n(d_rois, d_wle, d_n, 20000, sh)
    r = qlib.RenderContext(para, capacity=40000)
    r.render_device(loc.device_rows(), loc.device_valid_num(), 40000, stream=sh)
    img = r.read(sh)[0]
    rows, _ = loc.read_rows(sh)
    assert rows.shape[0] > 500
    host = qlib.RenderContext(para, capacity=40000)
    host.render(rows)
    close(img, host.read()[0])
    close(img, O.render(para, rows, 0)[0])
    assert img.sum() > 0
    for c in (r, host, loc, ex):
        c.close()
