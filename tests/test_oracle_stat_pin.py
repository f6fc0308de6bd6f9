"""The oracle's localization statistics (oracle/qcs_oracle_stat.c) pinned bit
for bit to the reference's own FluoStatisticData_TypeDef built for the host
(oracle/_ref): the four histograms and every mean after each call, over
several calls (the time-series means), 2D and 3D (neighbour radius 10 or 20
px), multi-emitter fitting on and off (density correction), and a call with
too few rows for a density (kept from before)."""
import numpy as np
import pytest

import oracle_lib as O
from qcstorm_b200.abi import default_para
from qcstorm_b200.synth import blinking_rows, group_sizes

pytestmark = pytest.mark.skipif(O.ref_host() is None, reason="reference host build absent")


@pytest.mark.parametrize("loc_type,multi", [(0, 0), (0, 1), (1, 0)])
def test_stat_oracle_matches_reference_host_build(loc_type, multi):
    rows, counts = blinking_rows(n_emitters=2000, frames=24, seed=7 + loc_type, width=512, loc_type=loc_type)
    rows[::97, 9] = 80.0   # some rows outside the precision window
    rows[::89, 6] = 10.0   # and below the photon floor
    sizes = list(group_sizes(counts, 6)) + [20]
    rows = np.concatenate([rows, rows[:20]])
    para = default_para(LocType=loc_type, MultiEmitterFitEn=multi, ImageWidth=512, ImageHigh=512, PixelSize=100.0)
    h_ref, m_ref = O.stat(para, rows, sizes, lib="ref")
    h_ora, m_ora = O.stat(para, rows, sizes, lib="oracle")
    np.testing.assert_array_equal(h_ora, h_ref)
    np.testing.assert_array_equal(m_ora.view(np.uint32), m_ref.view(np.uint32))
    assert h_ref[0].sum() > 1000 and m_ref[0, 6] > 0


def test_ontime_oracle_matches_reference_host_build():
    """UpdateOntimeRatio: the exponential fit's mean on time and the folded,
    clamped ratios, bit for bit (NaN where the reference gives NaN), on noisy
    decays, normalised decays, flat and rising ratios and degenerate starts."""
    rng = np.random.default_rng(41)
    cases = []
    for k in range(300):
        a, b = rng.uniform(0.05, 1.0), -rng.uniform(0.02, 4.0)
        y = a * np.exp(b * np.arange(10)) * (1 + rng.normal(0, 0.2, 10))
        cases.append(y / y.sum() if k % 3 == 0 else y)
    cases += [rng.uniform(0, 1, 10) for _ in range(40)]
    cases += [np.zeros(10), np.r_[0.01, 0.01, np.zeros(8)], np.r_[0.011, 0.02, np.zeros(8)], np.ones(10)]
    r = np.asarray(cases, np.float32)
    m_ref, s_ref = O.ontime(r, lib="ref")
    m_ora, s_ora = O.ontime(r, lib="oracle")
    np.testing.assert_array_equal(m_ora.view(np.uint32), m_ref.view(np.uint32))
    np.testing.assert_array_equal(s_ora.view(np.uint32), s_ref.view(np.uint32))
    assert np.isfinite(m_ref).sum() > 250
