"""The autotuner (qcs_loc_autotune): per batch size, the fastest of one
thread per ROI and the lane-group kernel (4, 8, 16 lanes for GS2D 7x7; 8 for
the other shapes) is kept in the context, and localizations with a tuned
context give the untuned rows bit for bit (the kernels' rows are identical),
for a table forcing every lane count and for the measured one."""
import numpy as np
import pytest

from qcstorm_b200 import lib as qlib
from qcstorm_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("gen,R,lanes", [(synth.gs2d_rois, 7, (1, 4, 8, 16)), (synth.as3d_rois, 9, (1, 8)),
                                         (synth.gs2d_rois, 11, (1, 8))])
def test_autotune_table_and_identical_rows(cuda_ok, gen, R, lanes):
    import torch
    rec, para, _ = gen(6000, R=R, seed=3)
    n = rec.shape[0]
    d = torch.from_numpy(rec.view(np.int16)).cuda()
    ctx = qlib.LocContext(para, capacity=n)
    wle = torch.from_numpy(ctx.wle(rec)).cuda()
    torch.cuda.synchronize()
    s = torch.cuda.Stream()
    ctx.localize_device(d.data_ptr(), n, wle.data_ptr(), s.cuda_stream)
    base, _ = ctx.read_rows(s.cuda_stream)
    table = ctx.autotune(d.data_ptr(), wle.data_ptr(), n, stream=s.cuda_stream)
    assert table and table[-1][0] >= n
    assert all(l in lanes for _, l in table)
    for m in (300, n):
        for l in lanes + (None,):
            if l is not None:
                ctx.set_tuning([(1 << 30, l)])
            else:
                ctx.set_tuning(table)
            ctx.localize_device(d.data_ptr(), m, wle.data_ptr(), s.cuda_stream)
            got, _ = ctx.read_rows(s.cuda_stream)
            np.testing.assert_array_equal(got.view(np.uint32), base[:m].view(np.uint32))
    with pytest.raises(RuntimeError):
        ctx.set_tuning([(100, 3)])
    ctx.close()
