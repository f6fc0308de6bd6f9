"""WLE pre-pass of a localization context with the conditional sort.

The nearest-neighbour search scans records in (frame, y, x) order.  A
context sorts the keys only when some record is out of that order (a CUDA
graph's IF node, condition set on the device); otherwise it scans the
records' own keys.  Both branches must give the rows of the reference's
all-pairs search: crowded frames (40 ROIs per frame within 200 px, so that
neighbour distances and molecule types vary) are given in order, shuffled,
reversed and with one swapped pair, with the batch smaller than and equal to
the context capacity.
"""
import numpy as np
import pytest

import oracle_lib as O
from qcstorm_b200 import lib as qlib
from qcstorm_b200 import synth

pytestmark = pytest.mark.gpu


def crowded(n, R, seed, per_frame=40):
    rec, para, _ = synth.gs2d_rois(n, R=R, seed=seed)
    rng = np.random.default_rng(seed)
    frames = 1 + np.arange(n) // per_frame
    xy = rng.integers(R, 200, size=(n, 2))
    rec[:, R * R + 0] = xy[:, 0]
    rec[:, R * R + 1] = xy[:, 1]
    rec[:, R * R + 2] = frames % 65536
    rec[:, R * R + 3] = frames // 65536
    order = np.lexsort((rec[:, R * R + 0], rec[:, R * R + 1], frames))
    return np.ascontiguousarray(rec[order]), para


def orders(n, seed):
    rng = np.random.default_rng(seed)
    swap = np.arange(n)
    swap[[n // 2, n // 2 + 1]] = swap[[n // 2 + 1, n // 2]]
    return {"sorted": np.arange(n), "shuffled": rng.permutation(n), "reversed": np.arange(n)[::-1].copy(),
            "one_swap": swap}


@pytest.mark.parametrize("n,capacity", [(3000, 3000), (2001, 5000)])
def test_wle_independent_of_record_order(cuda_ok, n, capacity):
    R = 7
    rec, para = crowded(n, R, seed=n)
    ctx = qlib.LocContext(para, capacity=capacity)
    base = ctx.wle(rec)
    ref = O.ref_gpu_wle(para, rec)
    assert np.array_equal(base.view(np.uint32), ref.view(np.uint32))
    assert (base[:, 0] < R).mean() > 0.05         # neighbours closer than the ROI size occur
    assert len(np.unique(base[:, 5])) > 1          # more than one molecule type
    for name, perm in orders(n, seed=1).items():
        got = ctx.wle(np.ascontiguousarray(rec[perm]))
        back = np.empty_like(got)
        back[perm] = got
        assert np.array_equal(back.view(np.uint32), base.view(np.uint32)), name
    ctx.close()


def test_localization_after_unsorted_batch(cuda_ok):
    """A sorted batch after an unsorted one on the same context (the sort's
    condition is reset at every call): rows equal a fresh context's."""
    R = 7
    rec, para = crowded(3000, R, seed=9)
    shuffled = np.ascontiguousarray(rec[np.random.default_rng(2).permutation(rec.shape[0])])
    ctx = qlib.LocContext(para, capacity=3000)
    ctx.localize(shuffled)
    rows, _ = ctx.localize(rec)
    fresh = qlib.LocContext(para, capacity=3000)
    rows0, _ = fresh.localize(rec)
    assert np.array_equal(rows.view(np.uint32), rows0.view(np.uint32))
    ctx.close()
    fresh.close()
