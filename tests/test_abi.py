"""C ABI: the library loads without a GPU, exports every declared symbol,
and mirrors the reference record layout."""
import ctypes
import os
import re

import numpy as np
import pytest

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


def test_batch_inputs_rejected_before_device_use():
    from andfn_b200 import _ffi
    from andfn_b200.records import layout_of
    L = _ffi.lib()
    g = load_golden("mixed")
    F, E = g["F_in"].copy(), g["E_in"].copy()
    lay = layout_of(E.dtype, F.dtype)
    h = ctypes.c_void_p()
    fp = (ctypes.c_void_p * 2)(F.ctypes.data, F.ctypes.data)
    ep = (ctypes.c_void_p * 2)(E.ctypes.data, E.ctypes.data)
    nf = np.array([len(F), 0], np.int64)  # second realization empty
    ne = np.array([len(E), len(E)], np.int64)
    rc = L.andfn_b200_batch_create(ctypes.byref(h), 2, fp, nf.ctypes.data_as(ctypes.c_void_p), ep,
                                   ne.ctypes.data_as(ctypes.c_void_p), ctypes.byref(lay), 50, -1)
    assert rc == 11 and "empty" in _ffi.last_error()
    rc = L.andfn_b200_batch_create(ctypes.byref(h), 0, fp, nf.ctypes.data_as(ctypes.c_void_p), ep,
                                   ne.ctypes.data_as(ctypes.c_void_p), ctypes.byref(lay), 50, -1)
    assert rc == 11
    assert L.andfn_b200_realizations(None) == 0


def test_memory_cache_accessors_without_device_use():
    """The device memory cache's accessors touch no device: an empty cache
    reports zero bytes, a device index out of range is rejected."""
    from andfn_b200 import _ffi
    import andfn_b200
    L = _ffi.lib()
    b = ctypes.c_int64(-1)
    assert L.andfn_b200_cached_memory(64, ctypes.byref(b), None, None) == 11
    assert L.andfn_b200_cached_memory(-1, ctypes.byref(b), None, None) == 11
    cm = andfn_b200.cached_memory(0)
    assert cm["bytes"] >= 0 and cm["hits"] >= 0 and cm["misses"] >= 0


def test_batch_records_must_share_dtypes():
    import andfn_b200
    from andfn_b200.records import element_dtype
    g = load_golden("mixed")
    F, E = g["F_in"].copy(), g["E_in"].copy()
    E2 = np.zeros(len(E), element_dtype(12))
    with pytest.raises(ValueError):
        andfn_b200.solve_batch([(F, E), (F.copy(), E2)], 50, g["constants_1"])


def test_record_structs_match_the_header(tmp_path):
    """Every struct of include/andfn_b200.h has the size and field offsets of
    its ctypes mirror in andfn_b200/records.py (gcc compiles a probe)."""
    import json
    import shutil
    import subprocess
    from andfn_b200 import records
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    names = ["AndfnLayout", "AndfnConstants", "AndfnSolveStats", "AndfnAdjointStats", "AndfnResidual"]
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "andfn_b200.h"', 'int main(void) {',
             'printf("{");']
    for k, n in enumerate(names):
        cls = getattr(records, n)
        lines.append(f'printf("{"," if k else ""}\\"{n}\\": [%zu", sizeof({n}));')
        for f, _ in cls._fields_:
            lines.append(f'printf(", %zu", offsetof({n}, {f}));')
        lines.append('printf("]");')
    lines += ['printf("}\\n");', "return 0;", "}"]
    src = tmp_path / "probe.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "probe"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = json.loads(subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout)
    for n in names:
        cls = getattr(records, n)
        want = [ctypes.sizeof(cls)] + [getattr(cls, f).offset for f, _ in cls._fields_]
        assert got[n] == want, (n, got[n], want)
