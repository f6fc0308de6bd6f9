"""The whole-frame pipeline captured in one CUDA graph: frames -> ROI
extraction -> (learned) multi-emitter localization -> CRLB -> render
hand-off, every step through the C ABI on one stream with no host
synchronisation, captured once and replayed.

The device-resident entry points enqueue kernels, memsets and copies only
(no allocation, no host wait), so a capture of one call sequence replays it:
the replayed rows equal the eagerly run rows bit for bit, and the rendered
image equals the eager image up to the order of its float atomic additions.
"""
import numpy as np
import pytest

from qcstorm_b200 import lib as qlib
from qcstorm_b200 import synth

pytestmark = pytest.mark.gpu

W = H = 512
NF = 4
CAP = 8000


def setup():
    import torch
    fr, para, _ = synth.frames(NF, width=W, height=H, density=300, seed=5)
    para.MultiEmitterFitEn = 1
    para.PixelZoom = 4.0
    para.SRImageWidth = (int(para.ImageWidth * para.PixelZoom) + 3) // 4 * 4
    para.SRImageHigh = (int(para.ImageHigh * para.PixelZoom) + 3) // 4 * 4
    d_fr = torch.from_numpy(fr.view(np.int16)).cuda()
    torch.cuda.synchronize()
    return fr, para, d_fr


def run_graph_case(net=None):
    import torch
    fr, para, d_fr = setup()
    ex = qlib.ExtractContext(para, max_batched_num=1, capacity=CAP)
    loc = qlib.LocContext(para, capacity=CAP)
    ren = qlib.RenderContext(para, capacity=2 * CAP)
    s = torch.cuda.Stream()
    sh = s.cuda_stream
    fb = W * H * 2
    d_rois, d_wle, d_n = ex.device_records()

    def step():
        ex.reset(sh)
        for f in range(NF):
            ex.extract_device(d_fr.data_ptr() + f * fb, 1, f, stream=sh)
        if net is None:
            loc.localize_device_n(d_rois, d_wle, d_n, CAP, sh)
        else:
            net.localize_n(loc, d_rois, d_wle, d_n, CAP, iters=2, bisections=6, stream=sh)
        ren.render_device(loc.device_rows(), loc.device_valid_num(), 2 * CAP, stream=sh)

    step()
    eager_rows, eager_ratios = loc.read_rows(sh)
    eager_img = ren.read(sh)[0]
    ren.reset(sh)
    s.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s, capture_error_mode="relaxed"):
        step()
    for _ in range(3):
        ren.reset(sh)
        with torch.cuda.stream(s):
            g.replay()
    graph_rows, graph_ratios = loc.read_rows(sh)
    graph_img = ren.read(sh)[0]
    assert eager_rows.shape[0] > 1000
    np.testing.assert_array_equal(graph_rows.view(np.uint32), eager_rows.view(np.uint32))
    np.testing.assert_array_equal(np.asarray(graph_ratios), np.asarray(eager_ratios))
    np.testing.assert_allclose(graph_img, eager_img, rtol=1e-4, atol=1e-3)
    assert graph_img.sum() > 0
    del g
    for c in (ren, loc, ex):
        c.close()
    return eager_rows


def test_frame_pipeline_in_a_cuda_graph(cuda_ok):
    run_graph_case()


def test_learned_frame_pipeline_in_a_cuda_graph(cuda_ok):
    """The same with the learned call (fused tensor-core inference with
    emitter-count classes, learned single-emitter stage, refits, 2E / 3E)."""
    import torch
    net = qlib.LearnedNet(batch=1024, seed=3)
    net.set_count_threshold(0.5)
    # an untrained network still exercises every kernel; its weight image is
    # built before the capture (the first call outside it)
    run_graph_case(net)
    net.fused_status()
    torch.cuda.synchronize()
    net.close()
