"""The render oracle (oracle/qcs_oracle_render.c) against the reference's own
render kernels built for the host (oracle/_ref/libqcs_ref_host.so:
FluoRenderWithPrec_2D / _3D run one emulated thread at a time, so rows are
added in row order, as the oracle adds them): images, z-weighted colour map,
display maximum and histogram equal bit for bit, for every rendering mode,
2D and 3D, in one call and accumulated over two."""
import numpy as np
import pytest

import oracle_lib as O
from render_rows import render_para, render_rows

pytestmark = pytest.mark.skipif(O.ref_host() is None, reason="reference host build absent")


def accumulated(p):
    """Empty images and an accumulated display maximum: while the maximum is 0
    (a first row whose splat centre is below 1) the reference's histogram
    step divides by it, which traps in the host build, so every case starts
    past that point."""
    shape = (p.SRImageHigh, p.SRImageWidth)
    return np.zeros(shape, np.float32), np.zeros(shape, np.float32), 1000, np.zeros(400, np.int32)


def equal(a, b):
    ia, ca, ma, ha = a
    ib, cb, mb, hb = b
    assert np.array_equal(ia.view(np.uint32), ib.view(np.uint32))
    assert np.array_equal(ca.view(np.uint32), cb.view(np.uint32))
    assert ma == mb
    assert np.array_equal(ha, hb)


@pytest.mark.parametrize("loc_type,mode", [(0, 0), (0, 1), (0, 2), (0, 3), (1, 0), (1, 1), (1, 2), (2, 0)])
def test_render_matches_reference_host_build(loc_type, mode):
    p = render_para(loc_type)
    rows = render_rows(3000, p, seed=7 + mode + 10 * loc_type)
    start = accumulated(p)
    ours = O.render(p, rows, mode, fixed_prec=12.5, state=start)
    ref = O.render(p, rows, mode, fixed_prec=12.5, state=start, lib="ref")
    equal(ours, ref)
    img = ours[0]
    assert img.sum() > 0 and ours[2] > 0 and ours[3].sum() > 0
    if loc_type != 0:
        assert np.abs(ours[1]).sum() > 0


def test_render_accumulates_like_reference():
    p = render_para(0)
    a, b = render_rows(1500, p, seed=1), render_rows(1500, p, seed=2)
    ours = O.render(p, b, 0, state=O.render(p, a, 0, state=accumulated(p)))
    ref = O.render(p, b, 0, state=O.render(p, a, 0, state=accumulated(p), lib="ref"), lib="ref")
    equal(ours, ref)
