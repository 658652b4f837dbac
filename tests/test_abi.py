"""C ABI: the library loads without a GPU, exports every declared symbol,
and mirrors the reference record layout."""
import ctypes
import os
import re

import numpy as np

from conftest import ROOT, load_golden


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "andfn_b200.h")).read()
    return sorted(set(re.findall(r"\b(andfn_b200_\w+)\s*\(", src)))


def test_library_exports_all_header_symbols():
    from andfn_b200 import _ffi
    L = _ffi.lib()
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, missing
    assert b"sm_100a" in L.andfn_b200_version()


def test_record_layout_matches_reference_defaults():
    from andfn_b200.records import element_dtype, fracture_dtype, layout_of
    E, F = element_dtype(200), fracture_dtype(500)
    assert E.itemsize == 12992 and F.itemsize == 4136
    lay = layout_of(E, F)
    # offsets of the reference's packed dtypes at MAX_NCOEF=200, MAX_ELEMENTS=500
    assert (lay.e_endpoints0, lay.e_ncoef, lay.e_q, lay.e_thetas, lay.e_coef, lay.e_old_coef,
            lay.e_dpsi_corr, lay.e_error, lay.e_error_coef) == (32, 136, 152, 160, 3360, 6560, 9760, 12960, 12984)
    assert (lay.f_elements, lay.f_nelements, lay.f_constant) == (120, 4120, 4128)


def test_golden_records_use_reference_field_order():
    from andfn_b200.records import element_dtype, fracture_dtype
    g = load_golden("c1_seed3")
    assert g["E_in"].dtype.names == element_dtype(10).names
    assert g["F_in"].dtype.names == fracture_dtype(10).names


def test_bad_layout_rejected_before_device_use():
    from andfn_b200 import _ffi
    from andfn_b200.records import AndfnLayout
    L = _ffi.lib()
    h = ctypes.c_void_p()
    lay = AndfnLayout()  # all zeros: invalid
    buf = np.zeros(64, np.uint8)
    rc = L.andfn_b200_create(ctypes.byref(h), buf.ctypes.data_as(ctypes.c_void_p), 1,
                             buf.ctypes.data_as(ctypes.c_void_p), 1, ctypes.byref(lay), 50, -1)
    assert rc == 10
    assert "layout" in _ffi.last_error()
