"""The torch generators (qcstorm_b200.synth_torch, used to make millions of
records on the GPU) against the numpy generators of the same workloads, on the
CPU: same record layout and header words, same parameters, and the same
distributions (means and spreads of the pixels and of every truth field within
sampling error)."""
import numpy as np
import pytest

from qcstorm_b200 import synth
from qcstorm_b200 import synth_torch as ST

GEN = {"gs2d": (synth.gs2d_rois, 7), "as3d": (synth.as3d_rois, 9), "multi": (synth.multi_rois, 11)}


@pytest.mark.parametrize("kind", ST.KINDS)
def test_torch_generator_matches_numpy_generator(kind):
    f, R = GEN[kind]
    n = 20000
    rt, tt = ST.rois(kind, n, R, seed=5, device="cpu", first_frame=70000)
    rn, _, tn = f(n, R=R, seed=5, first_frame=70000)
    a = rt.numpy().view(np.uint16)
    assert a.shape == rn.shape
    np.testing.assert_array_equal(a[:, R * R:], rn[:, R * R:])
    pa, pn = a[:, :R * R].astype(np.float64), rn[:, :R * R].astype(np.float64)
    assert abs(pa.mean() - pn.mean()) < 0.02 * pn.mean()
    assert abs(pa.std() - pn.std()) < 0.02 * pn.std()
    for key, w in tn.items():
        v = tt[key].numpy()
        assert v.shape == w.shape, key
        assert abs(np.nanmean(v) - np.nanmean(w)) < 0.03 * (np.nanstd(w) + 1e-9) * 10, key
        assert abs(np.nanstd(v) - np.nanstd(w)) < 0.05 * np.nanstd(w) + 1e-9, key
    assert bytes(ST.para(kind, R)) == bytes(f(1, R=R)[1])
    # reproducible from the seed
    r1, _ = ST.rois(kind, 100, R, seed=9, device="cpu")
    r2, _ = ST.rois(kind, 100, R, seed=9, device="cpu")
    assert np.array_equal(r1.numpy(), r2.numpy())
