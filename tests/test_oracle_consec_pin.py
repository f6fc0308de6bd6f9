"""The oracle's consecutive-frame merging (oracle/qcs_oracle_consec.c) pinned
bit for bit to the reference's own ConsecutiveFit_TypeDef built for the host
(oracle/_ref): the output rows of every call and the on-time ratios, over
several groups, for 2D and astigmatic 3D rows (their CRLB differs), a
threshold below one pixel (integer positions must coincide) and one of 2.5
pixels, and a last call that flushes everything."""
import numpy as np
import pytest

import oracle_lib as O
from consec_rows import consec_rows, group_sizes
from qcstorm_b200.abi import default_para

pytestmark = pytest.mark.skipif(O.ref_host() is None, reason="reference host build absent")


@pytest.mark.parametrize("loc_type,th_nm,fpg", [(0, 80.0, 3), (0, 250.0, 2), (1, 80.0, 4), (1, 250.0, 3)])
def test_consec_oracle_matches_reference_host_build(loc_type, th_nm, fpg):
    rows, counts = consec_rows(n_emitters=300, frames=12, seed=5 + loc_type, loc_type=loc_type)
    para = default_para(LocType=loc_type, ConsecFit_DistanceTh_nm=th_nm, PixelSize=100.0, QE=0.8)
    sizes = group_sizes(counts, fpg)
    ref, ref_on = O.consec(para, rows, sizes, lib="ref")
    ora, ora_on = O.consec(para, rows, sizes, lib="oracle", gpu_rounding=0)
    assert len(ref) == len(ora) == sizes.size
    merged = 0
    for a, b in zip(ora, ref):
        assert a.shape == b.shape
        np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32))
        merged += int((b[:, 0] == 0).sum())
    np.testing.assert_array_equal(ora_on.view(np.uint32), ref_on.view(np.uint32))
    assert merged > 50  # chains were found and their later rows removed
    assert sum(x.shape[0] for x in ref) == rows.shape[0]
