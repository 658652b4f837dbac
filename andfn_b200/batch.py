"""Batched realizations: R independent networks solved by one launch sequence.

A Monte-Carlo study of a fracture statistics solves many small networks; one
network of a few hundred fractures fills a small part of a B200, so the
batch API lays all realizations out side by side in HBM and runs every kernel
of an outer iteration over all of them.  Each realization keeps its own loop
state (iteration count, errors, convergence counter), its own factorised
discharge system and its own stopping test, so its result equals a separate
``andfn.hpc.hpc_solve.solve`` call (andfn/hpc/hpc_solve.py:55-257) on it.

All networks must share one record layout (the same element and fracture
dtypes, i.e. the same MAX_NCOEF / MAX_ELEMENTS).
"""
from __future__ import annotations

import ctypes
from typing import Sequence

import numpy as np

from . import _ffi
from .records import AndfnSolveStats, constants_struct, layout_of
from .solver import points_args


def _pointers(networks):
    fr = [f for f, _ in networks]
    el = [e for _, e in networks]
    if not networks:
        raise ValueError("empty batch")
    lay = layout_of(el[0].dtype, fr[0].dtype)
    for f, e in networks:
        if f.dtype != fr[0].dtype or e.dtype != el[0].dtype:
            raise ValueError("all realizations must share the record dtypes")
        for a in (f, e):
            if a.ndim != 1 or len(a) == 0 or not a.flags.c_contiguous or not a.flags.writeable:
                raise ValueError("records must be non-empty, 1-d, C-contiguous and writeable")
    R = len(networks)
    fp = (ctypes.c_void_p * R)(*[f.ctypes.data for f in fr])
    ep = (ctypes.c_void_p * R)(*[e.ctypes.data for e in el])
    nf = np.array([len(f) for f in fr], np.int64)
    ne = np.array([len(e) for e in el], np.int64)
    return lay, fp, ep, nf, ne


def solve_batch(networks: Sequence, discharge_int: int, constants) -> list[dict]:
    """Solves every (fractures, elements) pair in place; returns per-realization stats.

    Raises ``AndfnError`` for layout/input/CUDA problems and for a singular
    system in any realization; MAX_ITERATIONS and non-finite outcomes are
    reported per realization in ``stats[r]['status']`` like the reference,
    which only logs them.
    """
    networks = list(networks)
    lay, fp, ep, nf, ne = _pointers(networks)
    R = len(networks)
    cst = constants_struct(constants)
    st = (AndfnSolveStats * R)()
    rc = _ffi.lib().andfn_b200_batch_solve(R, fp, nf.ctypes.data_as(ctypes.c_void_p), ep,
                                          ne.ctypes.data_as(ctypes.c_void_p), ctypes.byref(lay),
                                          int(discharge_int), ctypes.byref(cst), st)
    _ffi.check(rc, ok=(0, 1, 2))
    return [s.as_dict() for s in st]


class BatchSolver:
    """R networks resident in HBM across solves (the batched handle API)."""

    def __init__(self, networks: Sequence, discharge_int: int = 50, device: int = -1):
        self.networks = list(networks)
        self.layout, self._fp, self._ep, nf, ne = _pointers(self.networks)
        self.R = len(self.networks)
        self._h = ctypes.c_void_p()
        _ffi.check(_ffi.lib().andfn_b200_batch_create(
            ctypes.byref(self._h), self.R, self._fp, nf.ctypes.data_as(ctypes.c_void_p), self._ep,
            ne.ctypes.data_as(ctypes.c_void_p), ctypes.byref(self.layout), int(discharge_int), int(device)))
        self.stats: list[dict] = []

    def close(self):
        if self._h:
            _ffi.lib().andfn_b200_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def reset(self):
        _ffi.check(_ffi.lib().andfn_b200_reset_state(self._h))

    def run(self, constants) -> list[dict]:
        cst = constants_struct(constants)
        st = (AndfnSolveStats * self.R)()
        rc = _ffi.lib().andfn_b200_batch_run(self._h, ctypes.byref(cst), st)
        self.stats = [s.as_dict() for s in st]
        _ffi.check(rc, ok=(0, 1, 2))
        return self.stats

    def download(self):
        """Writes every realization's results into its records in place."""
        _ffi.check(_ffi.lib().andfn_b200_batch_download(self._h, self._fp, self._ep))

    def stream(self) -> int:
        return int(_ffi.lib().andfn_b200_stream(self._h) or 0)

    def set_profiling(self, on: bool = True):
        _ffi.check(_ffi.lib().andfn_b200_set_profiling(self._h, 1 if on else 0))

    def kernel_times(self) -> dict:
        ms = np.zeros(5)
        n = np.zeros(5, np.int64)
        _ffi.check(_ffi.lib().andfn_b200_kernel_times(self._h, ms.ctypes.data_as(ctypes.c_void_p),
                                                     n.ctypes.data_as(ctypes.c_void_p), 5))
        names = ("eval_rhs", "trisolve", "eval_sweep", "update", "reduce")
        return {k: (float(ms[i]), int(n[i])) for i, k in enumerate(names)}

    def eval_heads(self, r: int, frac_idx, z) -> np.ndarray:
        """Heads of realization r (andfn/hpc/hpc_fracture.py:205-252)."""
        frac_idx, z = points_args(frac_idx, z)
        out = np.empty(len(z))
        _ffi.check(_ffi.lib().andfn_b200_batch_eval_heads(self._h, int(r), frac_idx.ctypes.data_as(ctypes.c_void_p),
                                                         z.ctypes.data_as(ctypes.c_void_p), len(z),
                                                         out.ctypes.data_as(ctypes.c_void_p)))
        return out
