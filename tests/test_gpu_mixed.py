"""Mixed-size localization (qcs_loc_localize_mixed_device): the single-emitter
fits of several calls of different ROI sizes run in one persistent launch
whose blocks pull tiles of any size from one work list.  Each entry's rows,
counters and fit ratios must equal its own qcs_loc_localize_device call's bit
for bit (those calls are pinned to the reference's CUDA build by the
reference-parity tests), with multi-emitter fitting on or off, with the WLE
pre-pass inside the call or given, and with empty entries."""
import numpy as np
import pytest

from qcstorm_b200 import lib as qlib
from qcstorm_b200 import synth

pytestmark = pytest.mark.gpu


def _entry(gen, n, R, seed):
    import torch
    rec, para, _ = gen(n, R=R, seed=seed)
    ctx = qlib.LocContext(para, capacity=max(rec.shape[0], 1))
    d = torch.from_numpy(rec.view(np.int16)).cuda()
    wle = torch.from_numpy(ctx.wle(rec)).cuda()
    return dict(ctx=ctx, d=d, wle=wle, n=rec.shape[0], para=para)


def _per_size(entries, stream):
    out = []
    for e in entries:
        e["ctx"].localize_device(e["d"].data_ptr(), e["n"], e["wle"].data_ptr(), stream)
        out.append(e["ctx"].read_rows(stream))
    return out


def _compare(entries, base, stream):
    for e, (rows, ratios) in zip(entries, base):
        got, got_ratios = e["ctx"].read_rows(stream)
        assert got.shape == rows.shape
        np.testing.assert_array_equal(got.view(np.uint32), rows.view(np.uint32))
        np.testing.assert_array_equal(got_ratios, ratios)


@pytest.mark.parametrize("with_wle", [True, False])
def test_mixed_rows_equal_per_size_calls(cuda_ok, with_wle):
    import torch
    entries = [_entry(synth.gs2d_rois, 20000, 7, 11), _entry(synth.gs2d_rois, 9000, 9, 12),
               _entry(synth.multi_rois, 12000, 11, 13), _entry(synth.as3d_rois, 7000, 9, 14),
               _entry(synth.as3d_rois, 3000, 7, 15), _entry(synth.gs2d_rois, 5000, 11, 16)]
    torch.cuda.synchronize()
    s = torch.cuda.Stream()
    base = _per_size(entries, s.cuda_stream)
    assert any(e["para"].MultiEmitterFitEn for e in entries)
    qlib.localize_mixed_device([(e["ctx"], e["d"].data_ptr(), e["n"], e["wle"].data_ptr() if with_wle else 0)
                                for e in entries], s.cuda_stream)
    _compare(entries, base, s.cuda_stream)
    # the same again (the work-list counter is reset by every call), in another entry order
    order = [2, 0, 5, 1, 4, 3]
    qlib.localize_mixed_device([(entries[i]["ctx"], entries[i]["d"].data_ptr(), entries[i]["n"],
                                 entries[i]["wle"].data_ptr()) for i in order], s.cuda_stream)
    _compare(entries, base, s.cuda_stream)
    for e in entries:
        e["ctx"].close()


def test_mixed_small_and_empty_entries(cuda_ok):
    """Entries shorter than one tile, and an empty one, beside a full one."""
    import torch
    entries = [_entry(synth.gs2d_rois, 5, 7, 21), _entry(synth.gs2d_rois, 31, 9, 22),
               _entry(synth.multi_rois, 700, 11, 23)]
    torch.cuda.synchronize()
    s = torch.cuda.Stream()
    base = _per_size(entries, s.cuda_stream)
    empty = _entry(synth.as3d_rois, 50, 9, 24)
    empty["ctx"].localize_device(empty["d"].data_ptr(), 0, empty["wle"].data_ptr(), s.cuda_stream)
    empty_rows, _ = empty["ctx"].read_rows(s.cuda_stream)
    assert empty_rows.shape[0] == 0
    qlib.localize_mixed_device([(e["ctx"], e["d"].data_ptr(), e["n"], e["wle"].data_ptr()) for e in entries] +
                               [(empty["ctx"], empty["d"].data_ptr(), 0, empty["wle"].data_ptr())], s.cuda_stream)
    _compare(entries, base, s.cuda_stream)
    got, _ = empty["ctx"].read_rows(s.cuda_stream)
    assert got.shape[0] == 0
    for e in entries + [empty]:
        e["ctx"].close()


def test_mixed_argument_errors(cuda_ok):
    """Refused before any device work: a context twice, a ROI size outside 7/9/11, records off a 4-byte
    boundary, likelihood-ratio selection, too many entries."""
    import torch
    a = _entry(synth.gs2d_rois, 100, 7, 31)
    b = _entry(synth.gs2d_rois, 100, 13, 32)
    c = _entry(synth.multi_rois, 100, 11, 33)
    torch.cuda.synchronize()
    with pytest.raises(qlib.QcsError) as ei:
        qlib.localize_mixed_device([(a["ctx"], a["d"].data_ptr(), a["n"]), (a["ctx"], a["d"].data_ptr(), a["n"])])
    assert ei.value.code == 1
    with pytest.raises(qlib.QcsError) as ei:
        qlib.localize_mixed_device([(a["ctx"], a["d"].data_ptr(), a["n"]), (b["ctx"], b["d"].data_ptr(), b["n"])])
    assert ei.value.code == 2
    with pytest.raises(qlib.QcsError) as ei:
        qlib.localize_mixed_device([(a["ctx"], a["d"].data_ptr() + 2, a["n"] - 1)])
    assert ei.value.code == 1
    c["ctx"].set_model_selection("lr", 0.0)
    with pytest.raises(qlib.QcsError) as ei:
        qlib.localize_mixed_device([(a["ctx"], a["d"].data_ptr(), a["n"]), (c["ctx"], c["d"].data_ptr(), c["n"])])
    assert ei.value.code == 1
    with pytest.raises(qlib.QcsError) as ei:
        qlib.localize_mixed_device([(a["ctx"], a["d"].data_ptr(), a["n"])] * 7)
    assert ei.value.code == 1
    for e in (a, b, c):
        e["ctx"].close()
