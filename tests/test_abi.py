"""The C-ABI library loads and exports every function include/*.h declares;
host-side argument checks reject bad input before any device work."""
import ctypes as C
import glob
import os
import re

import pytest

from qcstorm_b200 import abi
from qcstorm_b200 import lib as qlib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(qcs_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_library_exports_header():
    L = qlib.load()
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert set(qlib._SIGS) == names


def test_para_layout_matches_reference_class():
    # 39 fields of LocalizationPara, all 4-byte
    assert C.sizeof(abi.LocPara) == 39 * 4


def test_para_default_matches_reference_default():
    import oracle_lib as O
    ref = O.ref_host()
    if ref is None:
        pytest.skip("reference host build not present")
    a = abi.LocPara()
    ref.qcsref_default_para(C.byref(a))
    b = abi.LocPara()
    qlib.load().qcs_loc_para_default(C.byref(b))
    c = abi.default_para()
    assert a.as_dict() == b.as_dict() == c.as_dict()


def test_bad_roisize_rejected_before_device():
    L = qlib.load()
    p = abi.default_para(ROISize=8)
    h = C.c_void_p()
    assert L.qcs_loc_init(C.byref(p), C.byref(h)) == 2  # QCS_ERR_ROISIZE
    assert b"ROISize" in L.qcs_last_error()
    p = abi.default_para(LocType=7)
    assert L.qcs_loc_init(C.byref(p), C.byref(h)) == 1  # QCS_ERR_ARG


def test_no_device_fails_loudly():
    L = qlib.load()
    if L.qcs_device_available():
        pytest.skip("a CUDA device is present")
    p = abi.default_para()
    h = C.c_void_p()
    assert L.qcs_loc_init(C.byref(p), C.byref(h)) == 4  # QCS_ERR_CUDA
    assert b"no CPU fallback" in L.qcs_last_error()


def test_noalloc_argument_checks_before_device():
    # the allocation-free entry point refuses bad arguments before touching a device
    L = qlib.load()
    p = abi.default_para()
    args = (C.c_void_p(16), C.c_void_p(16))
    assert L.qcs_localize_noalloc(C.byref(p), *args, 8193, C.c_void_p(16), None, None) == 3  # capacity
    assert L.qcs_localize_noalloc(C.byref(p), *args, 16, C.c_void_p(20), None, None) == 1  # unaligned rows
    p.QE = 0.0
    assert L.qcs_localize_noalloc(C.byref(p), *args, 16, C.c_void_p(16), None, None) == 1  # QE


def test_model_selection_needs_a_context():
    L = qlib.load()
    assert L.qcs_loc_set_model_selection(None, 1, 0.0) == 1
    assert L.qcs_loc_model_selection(None, None, None) == 1
