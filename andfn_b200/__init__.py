"""B200-native drop-in for AnDFN's analytic-element solve.

``andfn_b200.solve`` replaces ``andfn.hpc.hpc_solve.solve`` (same signature,
same in-place record contract); ``install()`` makes ``andfn.DFN.solve`` use
it by rebinding the module-level name that andfn/dfn.py:21 imports and
andfn/dfn.py:1840 calls.
"""
from __future__ import annotations

from .hpc_solve import last_stats, solve
from .records import (AndfnConstants, AndfnLayout, AndfnSolveStats, constants_dtype, default_constants,
                      element_dtype, fracture_dtype, layout_of)
from .solver import Solver
from .batch import BatchSolver, solve_batch

__version__ = "0.1.0"

_saved = {}


def release_cached_memory():
    """Free the device memory the library keeps for reuse between handles."""
    from . import _ffi
    _ffi.lib().andfn_b200_release_cached_memory()


def cached_memory(device: int = 0) -> dict:
    """Bytes of device memory cached on ``device``, and the cache's hits and
    misses since the process started."""
    import ctypes
    from . import _ffi
    b, h, m = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
    _ffi.check(_ffi.lib().andfn_b200_cached_memory(device, ctypes.byref(b), ctypes.byref(h), ctypes.byref(m)))
    return {"bytes": b.value, "hits": h.value, "misses": m.value}


def install():
    """Route ``andfn.DFN.solve`` through the GPU solve."""
    import andfn.dfn as dfn_mod
    if "hpc_solve" not in _saved:
        _saved["hpc_solve"] = dfn_mod.hpc_solve
    dfn_mod.hpc_solve = solve


def uninstall():
    import andfn.dfn as dfn_mod
    if "hpc_solve" in _saved:
        dfn_mod.hpc_solve = _saved.pop("hpc_solve")


__all__ = ["solve", "install", "uninstall", "release_cached_memory", "cached_memory", "Solver", "BatchSolver", "solve_batch", "last_stats", "element_dtype", "fracture_dtype",
           "constants_dtype", "default_constants", "layout_of", "AndfnLayout", "AndfnConstants",
           "AndfnSolveStats"]
