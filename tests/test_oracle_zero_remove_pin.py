"""Zero-row removal oracle pinned against the reference's RemoveZeroLocalizations
built for the host (bfgsMLE_Loc_top/ZeroLocalizationsRemove.cu:21-186): kept
rows, their order and their count, with and without frame ordering."""
import numpy as np
import pytest

import oracle_lib as O
from qcstorm_b200 import synth

pytestmark = pytest.mark.skipif(O.ref_host() is None, reason="reference host build not present")


def localized_rows(seed=3, n=3000, frames=(100, 140)):
    rec, para, _ = synth.multi_rois(n, R=7, seed=seed)
    rng = np.random.default_rng(seed)
    rec[:, 49 + 2] = rng.integers(frames[0], frames[1], n)
    rec[:, 49 + 3] = 0
    wl = O.wle(para, rec)
    rows, _ = O.localize(para, rec, wl)
    return np.ascontiguousarray(rows, np.float32)


@pytest.mark.parametrize("sort,f0,f1", [(0, 0, 0), (1, 100, 139), (1, 105, 120), (1, 200, 210)])
def test_zero_remove_bit_exact(sort, f0, f1):
    rows = localized_rows()
    a = O.zero_remove(rows, sort, f0, f1, "oracle")
    b = O.zero_remove(rows, sort, f0, f1, "ref")
    assert a.shape == b.shape
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_zero_remove_edge_values():
    """Peak photons just above 1 (kept without sorting, dropped with it: the
    sorting path truncates to int first), negative frames, empty input."""
    rows = np.zeros((6, 12), np.float32)
    rows[:, 0] = [0.0, 1.0, 1.5, 2.0, 7.0, 3.0]
    rows[:, 11] = [5, 5, 5, 5, -1, 6]
    for sort in (0, 1):
        a = O.zero_remove(rows, sort, 5, 6, "oracle")
        b = O.zero_remove(rows, sort, 5, 6, "ref")
        assert np.array_equal(a, b)
    assert O.zero_remove(rows, 0, 0, 0)[:, 0].tolist() == [1.5, 2.0, 7.0, 3.0]
    assert O.zero_remove(rows, 1, 5, 6)[:, 0].tolist() == [2.0, 3.0]
    assert O.zero_remove(rows[:0], 1, 5, 6).shape == (0, 12)
