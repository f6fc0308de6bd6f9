"""The FP64 Fisher-matrix CRLB side output (qcs_crlb_fisher_fp64) against
its CPU oracle (oracle/qcs_oracle_fisher.c, itself pinned to closed forms and
to the reference's diagonal estimate in tests/test_oracle_fisher.py), on the
rows of real localization calls: GS2D 7x7, astigmatic 9x9 (with the z bound)
and the 1-3 emitter 11x11 cascade (appended second emitters placed at the ROI
centre).  Both sides compute in double; the results are stored as float, so
they agree to float rounding (relative 1e-6)."""
import numpy as np
import pytest

import oracle_lib as O
from qcstorm_b200 import lib as qlib
from qcstorm_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("gen,R", [(synth.gs2d_rois, 7), (synth.as3d_rois, 9), (synth.multi_rois, 11)])
def test_fisher_crlb_matches_oracle(cuda_ok, gen, R):
    rec, para, truth = gen(20000, R=R, seed=88 + R)
    ctx = qlib.LocContext(para, capacity=rec.shape[0])
    rows, _ = ctx.localize(rec)
    ctx.close()
    n = rec.shape[0]
    ours = qlib.crlb_fisher(para, rows, rec)
    want = O.crlb_fisher(para, rows, rec)
    assert np.array_equal(ours[:, 7], want[:, 7])
    ok = ours[:, 7] == 0
    assert ok.sum() >= 0.9 * (rows[:, 0] > 0).sum()
    np.testing.assert_allclose(ours[ok, :7], want[ok, :7], rtol=1e-6, atol=1e-6)
    if para.LocType == 1:
        assert np.all(ours[ok, 2] > 0)
    # rejected rows are skipped
    assert np.all(ours[rows[:, 0] <= 0, 7] == 1)
    # the bound of an efficient estimator: fitted x scatter vs the bound on accepted single rows
    if R != 11:
        acc = ok[:n]
        fx = rows[:n][acc, 1] + R // 2 - rec[acc, R * R].astype(np.float64)
        rmse = np.sqrt(np.mean((fx - truth["x"][acc]) ** 2)) * para.PixelSize
        crlb = np.sqrt(np.mean(ours[:n][acc, 0] ** 2))
        assert 0.9 < rmse / crlb < 1.6, (rmse, crlb)


def test_fisher_crlb_argument_checks(cuda_ok):
    _, para, _ = synth.gs2d_rois(4, R=7, seed=1)
    L = qlib.load()
    import ctypes as C
    bad = para.copy(QE=0.0)
    assert L.qcs_crlb_fisher_fp64(C.byref(bad), C.c_void_p(16), 4, None, 0, C.c_void_p(16), None) == 1
    assert L.qcs_crlb_fisher_fp64(C.byref(para.copy(ROISize=8)), C.c_void_p(16), 4, None, 0, C.c_void_p(16),
                                  None) == 2
    assert L.qcs_crlb_fisher_fp64(C.byref(para), None, 4, None, 0, None, None) == 1
