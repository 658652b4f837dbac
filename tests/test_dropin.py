"""The drop-in hook: andfn.DFN.solve calls the module-level name hpc_solve
bound at andfn/dfn.py:21; install() rebinds it to andfn_b200.solve.

Runs only where the reference source tree is available: its path comes from
the environment variable ANDFN_REFERENCE (the test is skipped when it is
unset).  The reference's model-building code needs pyvista/h5py/matplotlib,
which are stubbed here as the solve path never calls them.  The GPU solve
itself is replaced by a recorder, so the test needs no device; the records
that DFN.solve hands over are the consolidated records the golden fixtures
hold, which the GPU parity tests solve.
"""
import os
import sys
import types

import numpy as np
import pytest

REF = os.environ.get("ANDFN_REFERENCE", "")


def _import_andfn():
    if not REF or not os.path.isdir(os.path.join(REF, "andfn")):
        pytest.skip("reference source tree not available (set ANDFN_REFERENCE)")
    for name in ("pyvista", "h5py", "matplotlib", "matplotlib.colors", "matplotlib.tri", "matplotlib.pyplot"):
        sys.modules.setdefault(name, types.ModuleType(name))
    sys.modules["matplotlib.colors"].LinearSegmentedColormap = type(
        "LinearSegmentedColormap", (), {"from_list": staticmethod(lambda *a, **k: None)})
    sys.modules["matplotlib.tri"].Triangulation = object
    if REF not in sys.path:
        sys.path.insert(0, REF)
    os.environ.setdefault("NUMBA_CACHE_DIR", os.path.join(os.path.dirname(__file__), "golden", ".numba_cache"))
    import andfn
    return andfn


def test_install_routes_dfn_solve(monkeypatch):
    andfn = _import_andfn()
    import andfn.dfn as dfn_mod

    import andfn_b200
    from andfn_b200 import hpc_solve as hs
    calls = []

    def recorder(F, E, D, C, ntype=None):
        calls.append((F.dtype, E.dtype, D, int(C["MAX_ITERATIONS"])))
        return E
    orig = dfn_mod.hpc_solve
    andfn_b200.install()
    try:
        assert dfn_mod.hpc_solve is andfn_b200.solve
        monkeypatch.setattr(dfn_mod, "hpc_solve", recorder)
        f0 = andfn.Fracture("a", 1.0, 1.0, np.array([0.0, 0, 0]), np.array([0.0, 0, 1]), ncoef=5, nint=10)
        andfn.ConstantHeadLine("c", np.array([-0.5 + 0j, 0.5 + 0j]), 1.0, f0, 5, 10)
        d = andfn.DFN("t", MAX_ITERATIONS=7)
        d.add_fracture([f0])
        d.solve()
        assert len(calls) == 1 and calls[0][2] == 50 and calls[0][3] == 7
        # the records DFN.solve passes have the layout the C ABI reads
        lay = andfn_b200.layout_of(calls[0][1], calls[0][0])
        assert lay.elem_size == calls[0][1].itemsize
    finally:
        andfn_b200.uninstall()
    assert dfn_mod.hpc_solve is orig
    assert hs.solve is andfn_b200.solve
