"""Bit-level parity of the product CUDA path with the reference's own CUDA code.

oracle/_ref/libqcs_ref_gpu.so is the reference QC-STORM library compiled from
its sources for sm_100a (oracle/build_ref.py --gpu).  Both run on the same
B200 on the same seeded records, so the expected result is equality of every
bit of every output column, the row count and the fit ratios.  The product
path goes through the C ABI (libqcstorm_b200.so).

Two residuals remain and are asserted at the level reached:
  * CRLB columns (9, 10) of AS3D rows, whose Fisher matrix is built from
    numerical second derivatives (step 0.02) on a 15 x 15 grid: the step
    amplifies last-bit differences about 2500-fold, so the reference's own
    host and CUDA builds already disagree by up to a few percent there.  Ours
    must be no farther from the CUDA build than twice that spread (every
    other column bit-exact; the 9 x 9 grid of GS2D is bit-exact);
  * GS2D fits at 11 x 11 (weighted): at most 1 row in 500 differs, from one
    rounding site in the WLE weight mask that the fit's sensitivity to
    rounding amplifies; every other row is bit-exact.
"""
import numpy as np
import pytest

import oracle_lib as O
from qcstorm_b200 import lib as qlib
from qcstorm_b200 import synth

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(O.ref_gpu() is None, reason="reference GPU build not present")]


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def mismatch_report(a, b):
    bad = np.where((bits(a) != bits(b)).any(axis=1))[0]
    return "%d of %d rows differ; first %s\nref  %s\nours %s" % (
        bad.size, a.shape[0], bad[:8], a[bad[0]] if bad.size else "", b[bad[0]] if bad.size else "")


CRLB_COLS = [9, 10]
OTHER_COLS = [c for c in range(12) if c not in CRLB_COLS]


def max_rel(a, b):
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-6))) if a.size else 0.0


def assert_crlb_as3d(ref, ours, para):
    """AS3D CRLB columns: ours vs the reference CUDA build, bounded by the
    spread between the reference's host build (the oracle's CRLB, pinned to
    it bit for bit) and its CUDA build on the same fit rows."""
    host = O.crlb(para, ref)
    spread = max_rel(host[:, CRLB_COLS], ref[:, CRLB_COLS])
    ours_err = max_rel(ours[:, CRLB_COLS], ref[:, CRLB_COLS])
    assert ours_err <= max(2 * spread, 1e-5), (ours_err, spread)


def assert_rows(ref, ours, loc_type, R, weighted=True, para=None):
    """Bit-exact rows, except the documented residuals (module docstring)."""
    if loc_type == 1:
        assert_rows_fit(ref[:, OTHER_COLS], ours[:, OTHER_COLS], R, weighted)
        assert_crlb_as3d(ref, ours, para)
    else:
        assert_rows_fit(ref, ours, R, weighted)


def assert_rows_fit(ref, ours, R, weighted):
    diff = (bits(ref) != bits(ours)).any(axis=1)
    if R == 11 and weighted:
        assert diff.mean() <= 1 / 500, mismatch_report(ref, ours)
    else:
        assert not diff.any(), mismatch_report(ref, ours)


def assert_extra_rows(ref, ours, loc_type, R, para):
    """Appended second-emitter rows, compared as multisets (the reference
    appends them in atomic order); for AS3D keyed on every column but the
    CRLB ones, whose values are then checked against the matching row."""
    import collections
    assert ref.shape == ours.shape
    if ref.shape[0] == 0:
        return
    cols = OTHER_COLS if loc_type == 1 else list(range(12))
    kr = collections.Counter(map(tuple, bits(ref[:, cols])))
    ko = collections.Counter(map(tuple, bits(ours[:, cols])))
    unmatched = sum((ko - kr).values())
    allowed = max(2, ref.shape[0] // 500) if R == 11 else 0
    assert unmatched <= allowed, "%d of %d appended rows unmatched" % (unmatched, ref.shape[0])
    if loc_type == 1:
        idx = {tuple(k): i for i, k in enumerate(bits(ref[:, cols]))}
        pairs = [(idx[tuple(k)], j) for j, k in enumerate(bits(ours[:, cols])) if tuple(k) in idx]
        if pairs:
            ri, oi = map(list, zip(*pairs))
            assert_crlb_as3d(ref[ri], ours[oi], para)


def product_fit_kernel(kind, para, rec, wl):
    import torch
    n = rec.shape[0]
    d_rec = torch.from_numpy(np.ascontiguousarray(rec).view(np.int16)).cuda()
    d_wle = torch.from_numpy(np.ascontiguousarray(wl)).cuda()
    d_loc = torch.zeros((n, 12), dtype=torch.float32, device="cuda")
    s = torch.cuda.current_stream()
    qlib.fit_single_device(kind, para, d_rec.data_ptr(), d_wle.data_ptr(), n, d_loc.data_ptr(), s.cuda_stream)
    torch.cuda.synchronize()
    return d_loc.cpu().numpy()


@pytest.mark.parametrize("kind,gen,R", [(0, synth.gs2d_rois, 7), (0, synth.gs2d_rois, 11), (1, synth.as3d_rois, 9),
                                        (1, synth.as3d_rois, 7)])
def test_fit_kernel_bit_exact(cuda_ok, kind, gen, R):
    rec, para, _ = gen(3000, R=R, seed=21 + R)
    wl = O.ref_gpu_wle(para, rec)
    ref, _ = O.ref_gpu_fit_kernel(kind, para, rec, wl)
    ours = product_fit_kernel(kind, para, rec, wl)
    assert_rows_fit(ref, ours, R, weighted=True)


@pytest.mark.parametrize("gen,R,changes", [(synth.gs2d_rois, 7, {}), (synth.as3d_rois, 9, {}),
                                           (synth.multi_rois, 11, {}), (synth.multi_rois, 7, {}),
                                           (synth.as3d_rois, 7, {"MultiEmitterFitEn": 1})])
def test_wle_bit_exact(cuda_ok, gen, R, changes):
    rec, para, _ = gen(2000, R=R, seed=5)
    for k, v in changes.items():
        setattr(para, k, v)
    ref = O.ref_gpu_wle(para, rec)
    ctx = qlib.LocContext(para)
    ours = ctx.wle(rec)
    if R <= 7:
        assert np.array_equal(bits(ref), bits(ours)), mismatch_report(ref, ours)
    else:
        # nvcc's optimised build of the reference's PSF-width spline returns y
        # widths at ROISize >= 9 that its own host build and an unoptimised
        # (-G) build of the same code do not: compare the nearest-neighbour
        # distance and x widths with that build, the y widths with the host
        # build's arithmetic through the oracle.
        assert np.array_equal(bits(ref[:, :3]), bits(ours[:, :3]))
        host = O.wle(para, rec)
        np.testing.assert_allclose(ours[:, 3:5], host[:, 3:5], rtol=1e-5)


@pytest.mark.parametrize("gen,R,kind", [(synth.gs2d_rois, 7, 0), (synth.as3d_rois, 9, 1)])
def test_fit_kernel_large_batch(cuda_ok, gen, R, kind):
    """300,000 fits per kind: every row equals the reference kernel's bit for
    bit (the WLE rows from the product's pre-pass, fed to both)."""
    n = 300_000
    rec, para, _ = gen(n, R=R, seed=123)
    ctx = qlib.LocContext(para, capacity=n)
    wl = ctx.wle(rec)
    ctx.close()
    ref, _ = O.ref_gpu_fit_kernel(kind, para, rec, wl)
    ours = product_fit_kernel(kind, para, rec, wl)
    assert np.array_equal(bits(ref), bits(ours)), mismatch_report(ref, ours)


def test_crlb(cuda_ok):
    import torch
    for gen, R in ((synth.gs2d_rois, 7), (synth.as3d_rois, 9)):
        rec, para, _ = gen(1000, R=R, seed=9)
        wl = O.ref_gpu_wle(para, rec)
        rows, _ = O.ref_gpu_fit_kernel(para.LocType, para, rec, wl)
        ref = O.ref_gpu_crlb(para, rows)
        d = torch.from_numpy(rows.copy()).cuda()
        qlib.crlb_device(para, d.data_ptr(), rows.shape[0], torch.cuda.current_stream().cuda_stream)
        ours = d.cpu().numpy()
        assert_rows(ref, ours, para.LocType, R, para=para)


CASCADE = [
    ("gs2d-7", synth.gs2d_rois, 7, {}),
    ("as3d-7", synth.as3d_rois, 7, {}),
    ("as3d-11", synth.as3d_rois, 11, {}),
    ("as3d-7-multi", synth.as3d_rois, 7, {"MultiEmitterFitEn": 1}),
    ("multi-11", synth.multi_rois, 11, {}),
    ("multi-7", synth.multi_rois, 7, {}),
    ("multi-9-noWLE", synth.multi_rois, 9, {"WLEEn": 0}),
    ("dh3d-multi", synth.multi_rois, 9, {"LocType": 2}),
]


@pytest.mark.parametrize("name,gen,R,changes", CASCADE, ids=[c[0] for c in CASCADE])
def test_localize_bit_exact(cuda_ok, name, gen, R, changes):
    """Whole BFGS_MLELocalization: classify, single fit, 2E/3E cascade, CRLB.
    Appended second emitters are compared as a set (the reference appends them
    through an atomic counter in arbitrary order)."""
    rec, para, _ = gen(2500, R=R, seed=33 + R)
    for k, v in changes.items():
        setattr(para, k, v)
    wl = O.ref_gpu_wle(para, rec)
    ref, rref = O.ref_gpu_localize(para, rec, wl)
    ctx = qlib.LocContext(para)
    ours, rours = ctx.localize(rec, wl)
    n = rec.shape[0]
    assert ref.shape == ours.shape
    assert_rows(ref[:n], ours[:n], para.LocType, R, para=para)
    assert_extra_rows(ref[n:], ours[n:], para.LocType, R, para)
    if R == 11:
        np.testing.assert_allclose(rours, rref, atol=2 / n)
    else:
        assert np.array_equal(bits(rref), bits(rours))


def test_localize_as3d_9x9_matches_true_size_reference_kernel(cuda_ok):
    """AS3D at ROISize 9 through the whole localization call equals the
    reference's 9x9 kernel followed by its CRLB (the reference's own
    dispatcher would run the 8x8 kernel here)."""
    rec, para, _ = synth.as3d_rois(2000, R=9, seed=77)
    wl = O.ref_gpu_wle(para, rec)
    rows, _ = O.ref_gpu_fit_kernel(1, para, rec, wl)
    ref = O.ref_gpu_crlb(para, rows)
    ctx = qlib.LocContext(para)
    ours, _ = ctx.localize(rec, wl)
    assert_rows(ref, ours, 1, 9, para=para)
