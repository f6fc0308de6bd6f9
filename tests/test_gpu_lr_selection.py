"""Likelihood-ratio model selection (qcs_loc_set_model_selection,
QCS_SELECT_LR) on the 1-3 emitter 11x11 workload, next to the reference's
SNR cascade (QCS_SELECT_CASCADE, the parity mode).

Every record is fitted with one, two and three emitters and keeps the
smallest accepted model unless a larger one raises 2 ln L (FP64) by more than
the threshold per added emitter.  Checked: the layout of the rows (each
record's own row, appended second emitters of distinct records); with an
infinite threshold each record keeps its one-emitter fit when that fit is
accepted, bit for bit the single-emitter kernel's row (whose acceptance the
multi-emitter width bound narrows); against the
generator's truth, the selection finds more of the second emitters of 2- and
3-emitter records than the cascade at equal or better position RMSE.  Run as
a script, the module prints the emitter-count confusion of both modes for a
range of thresholds."""
import json

import numpy as np
import pytest

from qcstorm_b200 import lib as qlib
from qcstorm_b200 import synth

R = 11


def per_record(rows, n, first_frame=1):
    own, extra = rows[:n], rows[n:]
    count = (own[:, 0] > 0).astype(np.int64)
    rec = extra[:, 11].astype(np.int64) - first_frame
    assert np.all((rec >= 0) & (rec < n)) and np.unique(rec).size == rec.size
    count[rec] += 1
    return count, rec


def truth_match(rows, rec, truth, n, radius=1.0):
    """Distance of every localization to the nearest true emitter of its record (px)."""
    frames = rows[:, 11].astype(np.int64) - 1
    ok = rows[:, 0] > 0
    fx = rows[ok, 1] + R // 2 - rec[frames[ok], R * R].astype(np.float64)
    fy = rows[ok, 2] + R // 2 - rec[frames[ok], R * R + 1].astype(np.float64)
    tx, ty = truth["x"][frames[ok]], truth["y"][frames[ok]]
    d = np.nanmin(np.hypot(fx[:, None] - tx, fy[:, None] - ty), axis=1)
    m = d < radius
    return {"localizations": int(ok.sum()), "matched": int(m.sum()),
            "rmse_px": float(np.sqrt(np.mean(d[m] ** 2)))}


def run(mode, th, n=20000, seed=611):
    rec, para, truth = synth.multi_rois(n, R=R, seed=seed)
    ctx = qlib.LocContext(para, capacity=n)
    if mode == "lr":
        ctx.set_model_selection("lr", th)
    rows, ratios = ctx.localize(rec)
    ctx.close()
    count, _ = per_record(rows, n)
    conf = np.zeros((3, 3), np.int64)
    np.add.at(conf, (truth["k"] - 1, count), 1)
    return rows, ratios, conf, truth_match(rows, rec, truth, n), rec, para


pytestmark = pytest.mark.gpu


def test_lr_selection_against_cascade(cuda_ok):
    _, _, conf_c, acc_c, _, _ = run("cascade", 0.0)
    rows, ratios, conf_l, acc_l, _, _ = run("lr", 0.0)
    assert ratios[0] == ratios[1] == ratios[2] == 1.0  # every record fitted with 1, 2 and 3 emitters
    assert abs(ratios[3] + ratios[4] + ratios[5] + ratios[6] - 1.0) < 1e-5
    second_c = conf_c[1:, 2].sum()  # 2- and 3-emitter records given a second localization
    second_l = conf_l[1:, 2].sum()
    assert second_l > 2 * second_c, (conf_c.tolist(), conf_l.tolist())
    assert conf_l[0, 2] <= 0.05 * conf_l[0].sum()  # few single-emitter records split in two
    assert acc_l["matched"] > acc_c["matched"]
    assert acc_l["rmse_px"] <= 1.02 * acc_c["rmse_px"], (acc_l, acc_c)


def test_infinite_threshold_keeps_accepted_single_fits(cuda_ok):
    import torch
    rows, _, _, _, rec, para = run("lr", 1e30)
    n = rec.shape[0]
    d = torch.from_numpy(rec.view(np.int16)).cuda()
    ctx = qlib.LocContext(para, capacity=n)
    wle = torch.from_numpy(ctx.wle(rec)).cuda()
    ctx.close()
    single = torch.zeros((n, 12), dtype=torch.float32, device="cuda")
    qlib.fit_single_device(0, para, d.data_ptr(), wle.data_ptr(), n, single.data_ptr(), 0)
    qlib.crlb_device(para, single.data_ptr(), n, 0)
    torch.cuda.synchronize()
    s = single.cpu().numpy()
    # the kernel-level fit runs with multi-emitter fitting off, whose width bound is R / 1.5 / 2.35; with it
    # on the fit also needs sigma <= R / 2 / 2.35 (bfgsMLE_GS2D_core.h:263)
    acc = (s[:, 0] > 0) & (s[:, 4] <= R / 2.0 / 2.35)
    assert acc.mean() > 0.5
    assert np.array_equal(rows[:n][acc].view(np.uint32), s[acc].view(np.uint32))


def test_model_selection_arguments(cuda_ok):
    _, para, _ = synth.multi_rois(16, R=R, seed=1)
    ctx = qlib.LocContext(para, capacity=16)
    assert ctx.model_selection()[0] == "cascade"
    with pytest.raises(qlib.QcsError):
        qlib.check(qlib.load().qcs_loc_set_model_selection(ctx.h, 5, 0.0))
    with pytest.raises(qlib.QcsError):
        ctx.set_model_selection("lr", -1.0)
    ctx.set_model_selection("lr", 0.0)
    assert ctx.model_selection() == ("lr", 10.0)
    ctx.set_model_selection("cascade")
    ctx.close()


if __name__ == "__main__":
    out = {}
    _, _, conf, acc, _, _ = run("cascade", 0.0, n=50000, seed=612)
    out["cascade"] = {"confusion": conf.tolist(), "accuracy": acc}
    for th in (5.0, 10.0, 20.0, 40.0, 80.0, 160.0):
        _, ratios, conf, acc, _, _ = run("lr", th, n=50000, seed=612)
        out["lr_%g" % th] = {"confusion": conf.tolist(), "accuracy": acc, "kept_1_2_3": [float(x) for x in ratios[3:6]]}
    print(json.dumps(out, indent=1))
