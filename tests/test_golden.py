"""Golden fixtures (tests/golden/, made by tests/golden/make_golden.py from the
reference's own code): each holds its inputs, the parameter struct and the
reference's outputs, so these checks need neither the reference tree nor its
builds.  ref_host_*: the reference compiled for the host; the CPU oracle equals
it bit for bit.  ref_gpu_*: the reference's CUDA built for sm_100a; the product
kernels equal it bit for bit (fits, CRLB, WLE at 7x7; the multi-emitter cascade
with appended rows compared as a set, their order being the reference's atomic
arrival order)."""
import glob
import os

import numpy as np
import pytest

import oracle_lib as O
from qcstorm_b200.abi import LocPara

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    path = os.path.join(HERE, name + ".npz")
    if not os.path.exists(path):
        pytest.skip("fixture %s not generated" % name)
    return np.load(path)


def para(z):
    return LocPara.from_buffer_copy(z["para"].tobytes())


def same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape and a.dtype == b.dtype
    assert np.array_equal(a.view(np.uint8), b.view(np.uint8))


def test_fixtures_present():
    assert len(glob.glob(os.path.join(HERE, "ref_host_*.npz"))) >= 8


@pytest.mark.parametrize("name", ["gs2d7", "as3d7", "multi11"])
def test_oracle_localize_equals_reference_host(name):
    z = load("ref_host_localize_" + name)
    p = para(z)
    same(O.wle(p, z["rois"]), z["wle"])
    rows, ratios = O.localize(p, z["rois"], z["wle"])
    same(rows, z["rows"])
    same(ratios, z["ratios"])


def test_oracle_fit_as3d9_equals_reference_host():
    """AS3D 9x9 at the kernel level (the reference's dispatcher would run its
    8x8 kernel at this size)."""
    z = load("ref_host_fit_as3d9")
    p = para(z)
    same(O.wle(p, z["rois"]), z["wle"])
    same(O.fit_single(1, p, z["rois"], z["wle"]), z["fit"])


def test_oracle_zero_remove_equals_reference_host():
    z = load("ref_host_zero_remove_gs2d7")
    same(O.zero_remove(z["rows"], 1, int(z["first"]), int(z["end"])), z["kept"])


def test_oracle_extract_equals_reference_host():
    z = load("ref_host_extract")
    ro, wo, f0, f1 = O.extract(para(z), z["frames"], int(z["batch"]))
    same(ro, z["rois"])
    same(wo, z["wle"])
    assert (f0, f1) == (int(z["first"]), int(z["end"]))


@pytest.mark.parametrize("kind", ["2d", "3d"])
def test_oracle_render_equals_reference_host(kind):
    z = load("ref_host_render_" + kind)
    p = para(z)
    shape = z["image"].shape
    start = (np.zeros(shape, np.float32), np.zeros(shape, np.float32), int(z["start_max"]), np.zeros(400, np.int32))
    img, cmap, mx, hist = O.render(p, z["rows"], 0, state=start)
    same(img, z["image"])
    same(cmap, z["colormap"])
    assert mx == int(z["max"])
    same(hist, z["hist"])


def test_oracle_ontime_equals_reference_host():
    z = load("ref_host_ontime")
    mean, shown = O.ontime(z["ratios"])
    same(mean, z["mean"])
    same(shown, z["shown"])
    assert np.isnan(z["mean"]).sum() >= 1 and np.isfinite(z["mean"]).sum() > 50


def product_fit(kind, p, rec, wl):
    import torch
    from qcstorm_b200 import lib as qlib
    n = rec.shape[0]
    d = torch.from_numpy(rec.view(np.int16)).cuda()
    w = torch.from_numpy(np.ascontiguousarray(wl)).cuda()
    out = torch.zeros((n, 12), dtype=torch.float32, device="cuda")
    qlib.fit_single_device(kind, p, d.data_ptr(), w.data_ptr(), n, out.data_ptr())
    fit = out.cpu().numpy()
    qlib.crlb_device(p, out.data_ptr(), n)
    return fit, out.cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("name,kind", [("gs2d7", 0), ("as3d9", 1)])
def test_product_fit_equals_reference_cuda(cuda_ok, name, kind):
    from qcstorm_b200 import lib as qlib
    z = load("ref_gpu_fit_" + name)
    p = para(z)
    fit, crlb = product_fit(kind, p, z["rois"], z["wle"])
    same(fit, z["fit"])
    if "crlb" in z:
        same(crlb, z["crlb"])
    wl = qlib.LocContext(p, capacity=z["rois"].shape[0]).wle(z["rois"])
    if p.ROISize <= 7:
        same(wl, z["wle"])
    else:  # y widths at ROISize >= 9: see test_wle_bit_exact
        same(wl[:, :3], z["wle"][:, :3])


@pytest.mark.gpu
def test_product_cascade_equals_reference_cuda(cuda_ok):
    from qcstorm_b200 import lib as qlib
    z = load("ref_gpu_localize_multi11")
    p = para(z)
    n = z["rois"].shape[0]
    ctx = qlib.LocContext(p, capacity=n)
    rows, ratios = ctx.localize(z["rois"], z["wle"])
    ctx.close()
    ref = z["rows"]
    assert rows.shape == ref.shape
    same(rows[:n], ref[:n])
    key = lambda a: a[np.lexsort(a.T[::-1])]
    same(key(rows[n:]), key(ref[n:]))
    same(ratios, z["ratios"])
