"""Localization file (qcs_locfile_*): rows appended as 12 float32 each, read
back the way the reference's loader reads them
(utility/Output file load and postprocessing/py_LoadBinaryLocData.py:
np.fromfile(path, dtype=np.float32).reshape(-1, 12)).  Host rows need no
GPU; rows queued from the device are in test_gpu_locfile_device below."""
import os
import tempfile

import numpy as np
import pytest

from qcstorm_b200 import lib as qlib


def rows(n, seed):
    return np.random.default_rng(seed).normal(size=(n, 12)).astype(np.float32)


def load(path):
    return np.fromfile(path, dtype=np.float32).reshape(-1, 12)


def test_host_rows_round_trip():
    a, b = rows(1000, 1), rows(37, 2)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "loc.bin")
        f = qlib.LocFile(path)
        f.write(a)
        f.write(b)
        f.write(np.zeros((0, 12), np.float32))
        assert f.rows() == 1037
        f.close()
        got = load(path)
        assert np.array_equal(got.view(np.uint32), np.concatenate([a, b]).view(np.uint32))
        g = qlib.LocFile(path, append=True)
        assert g.rows() == 1037
        g.write(a[:5])
        g.close()
        assert load(path).shape[0] == 1042
        h = qlib.LocFile(path)  # truncates
        h.close()
        assert os.path.getsize(path) == 0


def test_open_refuses_bad_path():
    with pytest.raises(RuntimeError):
        qlib.LocFile("/nonexistent-dir/loc.bin")


@pytest.mark.gpu
def test_device_rows_after_zero_removal(cuda_ok):
    """Localization -> zero-row removal on the device -> file, every count read
    on the device: the file holds the kept rows, in order, as the host path
    computes them; device and host appends keep their call order."""
    import torch
    from qcstorm_b200 import synth
    rec, para, _ = synth.gs2d_rois(20_000, seed=8)
    n = rec.shape[0]
    ctx = qlib.LocContext(para, capacity=n)
    d = torch.from_numpy(rec.view(np.int16)).cuda()
    s = torch.cuda.Stream()
    sh = s.cuda_stream
    ctx.localize_device(d.data_ptr(), n, 0, sh)
    z = qlib.ZeroRemover(capacity=2 * n)
    d_out = torch.empty((2 * n, 12), dtype=torch.float32, device="cuda")
    d_nv = torch.zeros(1, dtype=torch.int32, device="cuda")
    z.remove_device(ctx.device_rows(), 2 * n, d_out.data_ptr(), d_n=ctx.device_valid_num(), d_nvalid=d_nv.data_ptr(),
                    stream=sh)
    extra = rows(3, 9)
    with tempfile.TemporaryDirectory() as dd:
        path = os.path.join(dd, "loc.bin")
        f = qlib.LocFile(path, capacity=2 * n)
        f.write_device(d_out.data_ptr(), d_nv.data_ptr(), 2 * n, sh)
        f.write(extra)  # after the queued device rows
        f.write_device(d_out.data_ptr(), d_nv.data_ptr(), 2 * n, sh)
        f.flush()
        kept = int(d_nv.item())
        assert f.rows() == 2 * kept + 3
        f.close()
        got = load(path)
    plain, _ = ctx.read_rows(sh)
    exp = plain[plain[:, 0] > 1.0]
    assert kept == exp.shape[0] > 0.5 * n
    want = np.concatenate([exp, extra, exp])
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    ctx.close()
