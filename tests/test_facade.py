"""The reference-compatible C++ façade (include/qcstorm_b200.hpp): a program
written only against the reference's class names and member signatures
(tests/facade_check.cpp) compiles and links against libqcstorm_b200.so here,
and on a GPU gives the same records, rows and kept rows as the C ABI, and the
rendered image of the oracle's render within float summation order."""
import ctypes as C
import os
import subprocess
import tempfile

import numpy as np
import pytest

from qcstorm_b200 import lib as qlib
from qcstorm_b200 import synth
import oracle_lib as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.dirname(qlib.LIB_PATH)


def build(out_dir):
    exe = os.path.join(out_dir, "facade_check")
    cmd = ["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include",
           os.path.join(ROOT, "tests", "facade_check.cpp"), "-o", exe, "-L", LIBDIR, "-lqcstorm_b200",
           "-Wl,-rpath," + LIBDIR]
    if not os.path.exists(os.path.join(LIBDIR, "libcudart.so")):
        cmd += ["-L", "/usr/local/cuda/lib64", "-lcudart", "-Wl,-rpath,/usr/local/cuda/lib64"]
    subprocess.run(cmd, check=True, capture_output=True)
    return exe


def test_facade_compiles_and_links():
    with tempfile.TemporaryDirectory() as d:
        exe = build(d)
        assert os.path.exists(exe)


@pytest.mark.gpu
def test_facade_matches_c_abi(cuda_ok):
    fr, para, _ = synth.frames(4, width=256, height=192, density=120, seed=91)
    para.MultiEmitterFitEn = 1
    with tempfile.TemporaryDirectory() as d:
        exe = build(d)
        open(os.path.join(d, "para.bin"), "wb").write(bytes(para))
        np.ascontiguousarray(fr).tofile(os.path.join(d, "frames.bin"))
        open(os.path.join(d, "n_frames.txt"), "w").write("4")
        subprocess.run([exe, d], check=True, timeout=120)
        counts = list(map(int, open(os.path.join(d, "counts.txt")).read().split()))
        n, nloc, nkept, f0, f1, gf, gl = counts
        R = para.ROISize
        rois = np.fromfile(os.path.join(d, "rois.bin"), np.uint16).reshape(n, R * (R + 1))
        wle = np.fromfile(os.path.join(d, "wle.bin"), np.float32).reshape(n, 6)
        loc = np.fromfile(os.path.join(d, "loc.bin"), np.float32).reshape(nloc, 12)
        kept = np.fromfile(os.path.join(d, "kept.bin"), np.float32).reshape(nkept, 12)
        srw = (int(para.ImageWidth * para.PixelZoom) + 3) // 4 * 4
        srh = (int(para.ImageHigh * para.PixelZoom) + 3) // 4 * 4
        img = np.fromfile(os.path.join(d, "render.bin"), np.float32).reshape(srh, srw)
    batch = qlib.load().qcs_extract_max_batched_num(para.ImageWidth, para.ImageHigh)
    ro, wo, g0, g1 = O.extract(para, fr, batch, flags=O.EXTRACT_FMA_CONV | O.EXTRACT_EXACT_VARIANCE)
    assert np.array_equal(rois, ro) and (f0, f1) == (g0, g1) == (0, 3)
    ctx = qlib.LocContext(para)
    rows, _ = ctx.localize(rois, wle)
    ctx.close()
    assert np.array_equal(loc.view(np.uint32), rows.view(np.uint32))
    exp_kept = O.zero_remove(rows, 1, f0, f1)
    assert np.array_equal(kept.view(np.uint32), exp_kept.view(np.uint32))
    para.SRImageWidth, para.SRImageHigh = srw, srh
    exp_img = O.render(para, exp_kept, 0)[0]
    assert exp_img.sum() > 0
    np.testing.assert_allclose(img, exp_img, rtol=1e-4, atol=1e-3)  # atomic-add order, __expf
    frames = exp_kept[:, 11].astype(int)
    assert gf == next((f for f in frames if f != 0), 0)       # GetFirstFrame: first nonzero frame
    assert gl == next((f for f in frames[:0:-1] if f != 0), 0)  # GetLastFrame: last nonzero, row 0 excluded
