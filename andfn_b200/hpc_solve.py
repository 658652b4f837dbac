"""Drop-in replacement for ``andfn.hpc.hpc_solve.solve``.

``solve(fracture_struc_array, element_struc_array, discharge_int, constants,
ntype_elements)`` has the reference's signature and in-place contract
(andfn/hpc/hpc_solve.py:55-257): the element records get their coefficients,
ncoef/nint, thetas, q, errors and dpsi_corr updated, the fracture records get
their constants, and the element array is returned.  The work runs on a B200
through ``libandfn_b200.so``; there is no CPU path.

Error behaviour follows the reference where it has one: a singular discharge
system raises (SuperLU raises there, hpc_solve.py:121), hitting
MAX_ITERATIONS or producing NaN returns silently with a log line (the
reference only logs, hpc_solve.py:242-257).  Layout, input and CUDA problems
raise ``AndfnError``.
"""
from __future__ import annotations

import ctypes
import logging

import numpy as np

from . import _ffi
from .records import AndfnSolveStats, constants_struct, layout_of

logger = logging.getLogger("andfn")

last_stats: dict = {}


def _check_arrays(fracture_struc_array, element_struc_array):
    for name, a in (("fracture_struc_array", fracture_struc_array), ("element_struc_array", element_struc_array)):
        if not isinstance(a, np.ndarray) or a.dtype.fields is None:
            raise TypeError(f"{name} must be a numpy structured array")
        if not a.flags.c_contiguous or not a.flags.writeable:
            raise ValueError(f"{name} must be C-contiguous and writeable (it is updated in place)")
        if a.ndim != 1 or len(a) == 0:
            raise ValueError(f"{name} must be a non-empty 1-d array")


def solve(fracture_struc_array, element_struc_array, discharge_int, constants, ntype_elements=None):
    """Solve the DFN in place on the GPU; returns ``element_struc_array``."""
    _check_arrays(fracture_struc_array, element_struc_array)
    lay = layout_of(element_struc_array.dtype, fracture_struc_array.dtype)
    cst = constants_struct(constants)
    stats = AndfnSolveStats()
    L = _ffi.lib()
    logger.info("Solving on the GPU (andfn_b200)...")
    rc = L.andfn_b200_solve(fracture_struc_array.ctypes.data_as(ctypes.c_void_p), len(fracture_struc_array),
                            element_struc_array.ctypes.data_as(ctypes.c_void_p), len(element_struc_array),
                            ctypes.byref(lay), int(discharge_int), ctypes.byref(cst), ctypes.byref(stats))
    last_stats.clear()
    last_stats.update(stats.as_dict())
    _ffi.check(rc, ok=(0, 1, 2))
    logger.info("---------------------------------------")
    logger.info("Solver results")
    logger.info("---------------------------------------")
    logger.info(f"Iterations: {stats.iterations}, Error E: {stats.error:.3e}, Q: {stats.error_q:.3e}, ")
    logger.debug(f"GPU times (ms): setup {stats.ms_setup:.2f}, factor {stats.ms_factor:.2f}, "
                 f"iterate {stats.ms_iterate:.2f}, total {stats.ms_total:.2f}")
    if rc == 1:
        logger.info("Stopped at MAX_ITERATIONS before two converged rounds.")
    elif rc == 2:
        logger.warning("The solve produced non-finite coefficients or discharges.")
    return element_struc_array
