"""Localization statistics on the GPU (qcs_stat_*) against the CPU oracle
(pinned bit for bit to the reference's host build) and the reference's own
FluoStatisticData_TypeDef built for sm_100a (oracle/_ref): histograms and the
neighbour counts behind the activation density are integer results and equal
the oracle's exactly; the means come from float sums that the GPU adds in
another order (the reference's CUDA build with float atomics, this one per
block and then in block order), so they agree to float rounding; the time
series follow the calls; the device form equals the host form."""
import numpy as np
import pytest

import oracle_lib as O
from qcstorm_b200 import lib as qlib
from qcstorm_b200.abi import default_para
from qcstorm_b200.synth import blinking_rows, group_sizes

pytestmark = pytest.mark.gpu


def workload(loc_type, multi, seed=7):
    rows, counts = blinking_rows(n_emitters=2000, frames=24, seed=seed + loc_type, width=512, loc_type=loc_type)
    rows[::97, 9] = 80.0
    rows[::89, 6] = 10.0
    sizes = list(group_sizes(counts, 6)) + [20]
    rows = np.concatenate([rows, rows[:20]])
    para = default_para(LocType=loc_type, MultiEmitterFitEn=multi, ImageWidth=512, ImageHigh=512, PixelSize=100.0)
    return rows, sizes, para


def product(rows, sizes, para, device=False):
    import torch
    st = qlib.Statistics(capacity=int(max(sizes)))
    hs, ms = [], []
    o = 0
    for k in sizes:
        chunk = np.ascontiguousarray(rows[o:o + k])
        o += k
        if device:
            d = torch.from_numpy(chunk).cuda()
            torch.cuda.synchronize()
            h, m = st.update_device(d.data_ptr(), k, para)
        else:
            h, m = st.update(chunk, para)
        hs.append(h)
        ms.append(m)
    series = [st.series(i) for i in range(7)]
    st.close()
    return np.stack(hs), np.stack(ms), series


@pytest.mark.parametrize("loc_type,multi", [(0, 0), (0, 1), (1, 0)])
def test_stat_matches_oracle_and_reference(cuda_ok, loc_type, multi):
    rows, sizes, para = workload(loc_type, multi)
    h, m, series = product(rows, sizes, para)
    h_o, m_o = O.stat(para, rows, sizes, lib="oracle")
    np.testing.assert_array_equal(h, h_o)
    # density: integer neighbour counts, then the same float formula
    np.testing.assert_array_equal(m[:, 6].view(np.uint32), m_o[:, 6].view(np.uint32))
    # photon mean from the (equal) histograms
    np.testing.assert_array_equal(m[:, 0].view(np.uint32), m_o[:, 0].view(np.uint32))
    np.testing.assert_allclose(m, m_o, rtol=1e-5)
    assert len(series[0]) == len(sizes)
    np.testing.assert_allclose(series[0], m[:, 0])
    h_g, m_g = O.stat(para, rows, sizes, lib="ref_gpu")
    # the reference's CUDA build fuses sqrt(x^2 + y^2)'s products as nvcc chooses: a row at a bin edge may move
    assert np.abs(h.astype(np.int64) - h_g).sum() <= 4 * len(sizes)
    np.testing.assert_allclose(m, m_g, rtol=1e-4)


def test_stat_device_form_and_reset(cuda_ok):
    rows, sizes, para = workload(0, 0, seed=11)
    a = product(rows, sizes, para)
    b = product(rows, sizes, para, device=True)
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1].view(np.uint32), b[1].view(np.uint32))
    st = qlib.Statistics(capacity=int(max(sizes)))
    st.update(rows[:sizes[0]], para)
    st.reset()
    _, m = st.result()  # the host histograms keep the last call's, as the reference's do
    assert not m.any() and st.series(0).size == 0
    with pytest.raises(RuntimeError):
        st.update(np.zeros((int(max(sizes)) + 1, 12), np.float32), para)
    st.close()


def test_ontime_fit_equals_reference(cuda_ok):
    """qcs_stat_update_ontime_ratio against the reference's UpdateOntimeRatio
    (golden outputs of its host build, and the oracle pinned to it): mean on
    time and shown ratios bit for bit, call after call on one object; the four
    on-time series follow the shown ratios; a reset clears them and keeps the
    mean on time, as the reference does."""
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_host_ontime.npz"))
    st = qlib.Statistics(capacity=16)
    assert st.ontime()[0] == 0.0
    means, shown = [], []
    for r in z["ratios"]:
        m, s = st.update_ontime(r)
        means.append(m)
        shown.append(s)
    means = np.asarray(means, np.float32)
    shown = np.asarray(shown, np.float32)
    np.testing.assert_array_equal(means.view(np.uint32), z["mean"].view(np.uint32))
    np.testing.assert_array_equal(shown.view(np.uint32), z["shown"].view(np.uint32))
    for k in range(4):
        np.testing.assert_array_equal(st.series(qlib.STAT_SERIES_ONTIME_F1 + k), shown[:, k])
    last = st.ontime()[0]
    st.reset()
    assert st.series(qlib.STAT_SERIES_ONTIME_F1).size == 0
    assert np.asarray(st.ontime()[0], np.float32).view(np.uint32) == np.asarray(last, np.float32).view(np.uint32)
    with pytest.raises(ValueError):
        st.update_ontime(np.zeros(9, np.float32))
    st.close()


def test_ontime_from_consecutive_fit(cuda_ok):
    """The plug-ins' chain, ConsecutiveFit then UpdateOntimeRatio
    (OnlineLocalizationLD.cpp:312): the product's on-time ratios fed to the
    product's fit equal the oracle's fit of the same ratios."""
    rows, counts = blinking_rows(n_emitters=1500, frames=20, seed=77, width=512)
    para = default_para(LocType=0, ConsecFit_DistanceTh_nm=80.0, PixelSize=100.0, QE=0.8)
    sizes = group_sizes(counts, 4)
    cf = qlib.ConsecFit(capacity=int(max(sizes)))
    st = qlib.Statistics(capacity=16)
    o, ons = 0, []
    for g, k in enumerate(sizes):
        _, on = cf.fit(rows[o:o + k], para, is_end=g == len(sizes) - 1)
        o += k
        ons.append(on)
        m, s = st.update_ontime(on)
        m_o, s_o = O.ontime(on)
        assert np.float32(m).view(np.uint32) == m_o.view(np.uint32)[0]
        np.testing.assert_array_equal(s.view(np.uint32), s_o[0].view(np.uint32))
    assert np.isfinite(m) and 0.1 < m < 20.0
    cf.close()
    st.close()
