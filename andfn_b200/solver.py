"""Handle API: keep one network resident in HBM across solves.

``Solver`` wraps ``andfn_b200_create/run/download`` (include/andfn_b200.h).
It is what repeated solves (benchmarks, parameter sweeps, the adjoint) use,
so uploads and table construction happen once per network.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _ffi
from .records import AndfnSolveStats, constants_struct, layout_of


def points_args(frac_idx, z):
    """(frac_idx, z) as C-contiguous 1-d int64 / complex128 arrays of one
    length; the C entry points read len(z) entries of both."""
    frac_idx = np.ascontiguousarray(frac_idx, np.int64)
    z = np.ascontiguousarray(z, np.complex128)
    if frac_idx.ndim != 1 or z.ndim != 1 or frac_idx.shape != z.shape:
        raise ValueError(f"frac_idx and z must be 1-d arrays of one length (got shapes {frac_idx.shape} "
                         f"and {z.shape})")
    return frac_idx, z


def out_array(out, n, dtype=np.float64):
    """A caller's output array the C call writes n entries into: it must be a
    writeable, C-contiguous 1-d ndarray of dtype and length n (it cannot be
    converted, since the results must land in the caller's own array)."""
    if out is None:
        return np.empty(n, dtype)
    if (not isinstance(out, np.ndarray) or out.dtype != np.dtype(dtype) or out.ndim != 1 or out.shape[0] != n
            or not out.flags.c_contiguous or not out.flags.writeable):
        raise ValueError(f"out must be a writeable C-contiguous 1-d {np.dtype(dtype)} array of length {n}")
    return out


class Solver:
    def __init__(self, fractures: np.ndarray, elements: np.ndarray, discharge_int: int = 50, device: int = -1):
        if not (fractures.flags.c_contiguous and elements.flags.c_contiguous):
            raise ValueError("records must be C-contiguous")
        self.fractures, self.elements = fractures, elements
        self.layout = layout_of(elements.dtype, fractures.dtype)
        self._h = ctypes.c_void_p()
        L = _ffi.lib()
        _ffi.check(L.andfn_b200_create(ctypes.byref(self._h), fractures.ctypes.data_as(ctypes.c_void_p),
                                       len(fractures), elements.ctypes.data_as(ctypes.c_void_p), len(elements),
                                       ctypes.byref(self.layout), int(discharge_int), int(device)))
        self.stats: dict = {}

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

    def upload_state(self, fractures=None, elements=None):
        f = self.fractures if fractures is None else fractures
        e = self.elements if elements is None else elements
        _ffi.check(_ffi.lib().andfn_b200_upload_state(self._h, f.ctypes.data_as(ctypes.c_void_p),
                                                     e.ctypes.data_as(ctypes.c_void_p)))

    def reset(self):
        _ffi.check(_ffi.lib().andfn_b200_reset_state(self._h))

    def run(self, constants) -> dict:
        cst = constants_struct(constants)
        st = AndfnSolveStats()
        rc = _ffi.lib().andfn_b200_run(self._h, ctypes.byref(cst), ctypes.byref(st))
        self.stats = st.as_dict()
        _ffi.check(rc, ok=(0, 1, 2))
        return self.stats

    def download(self, fractures=None, elements=None):
        f = self.fractures if fractures is None else fractures
        e = self.elements if elements is None else elements
        _ffi.check(_ffi.lib().andfn_b200_download(self._h, f.ctypes.data_as(ctypes.c_void_p),
                                                 e.ctypes.data_as(ctypes.c_void_p)))
        return e

    KERNEL_CLASSES = ("eval_rhs", "trisolve", "eval_sweep", "update", "reduce")

    def set_profiling(self, on: bool = True):
        _ffi.check(_ffi.lib().andfn_b200_set_profiling(self._h, 1 if on else 0))

    def kernel_times(self) -> dict:
        ms = np.zeros(5)
        n = np.zeros(5, np.int64)
        _ffi.check(_ffi.lib().andfn_b200_kernel_times(self._h, ms.ctypes.data_as(ctypes.c_void_p),
                                                     n.ctypes.data_as(ctypes.c_void_p), 5))
        return {k: (float(ms[i]), int(n[i])) for i, k in enumerate(self.KERNEL_CLASSES)}

    def stream(self) -> int:
        return int(_ffi.lib().andfn_b200_stream(self._h) or 0)

    def eval_heads(self, frac_idx, z) -> np.ndarray:
        """Heads Re(Omega_f(z))/t_f (andfn/hpc/hpc_fracture.py:205-252)."""
        frac_idx, z = points_args(frac_idx, z)
        out = np.empty(len(z))
        _ffi.check(_ffi.lib().andfn_b200_eval_heads(self._h, frac_idx.ctypes.data_as(ctypes.c_void_p),
                                                   z.ctypes.data_as(ctypes.c_void_p), len(z),
                                                   out.ctypes.data_as(ctypes.c_void_p)))
        return out

    NOALLOC_MAX_POINTS = 65536

    def eval_heads_noalloc(self, frac_idx, z, out=None) -> np.ndarray:
        """Heads through the entry point that allocates no device memory
        (at most NOALLOC_MAX_POINTS points per call; calls on one device must
        not overlap in time).  Pass C-contiguous int64 / complex128 arrays and
        an out array (a writeable C-contiguous float64 array of len(z)) to
        avoid host-side copies as well."""
        frac_idx, z = points_args(frac_idx, z)
        out = out_array(out, len(z))
        _ffi.check(_ffi.lib().andfn_b200_eval_heads_noalloc(self._h, frac_idx.ctypes.data_as(ctypes.c_void_p),
                                                           z.ctypes.data_as(ctypes.c_void_p), len(z),
                                                           out.ctypes.data_as(ctypes.c_void_p)))
        return out

    def bc_residual(self) -> dict:
        """Boundary-condition residual per element and flux balance per
        fracture of the current state (include/andfn_b200.h)."""
        from .records import AndfnResidual
        res = np.empty(len(self.elements))
        flux = np.empty(len(self.fractures))
        out = AndfnResidual()
        _ffi.check(_ffi.lib().andfn_b200_bc_residual(self._h, res.ctypes.data_as(ctypes.c_void_p),
                                                    flux.ctypes.data_as(ctypes.c_void_p), ctypes.byref(out)))
        d = out.as_dict()
        d["elem"] = res
        d["flux"] = flux
        return d

    def eval_omega(self, frac_idx, z) -> np.ndarray:
        """Omega_f(z) (andfn/hpc/hpc_fracture.py:52-94)."""
        frac_idx, z = points_args(frac_idx, z)
        out = np.empty(len(z), np.complex128)
        _ffi.check(_ffi.lib().andfn_b200_eval_omega(self._h, frac_idx.ctypes.data_as(ctypes.c_void_p),
                                                   z.ctypes.data_as(ctypes.c_void_p), len(z),
                                                   out.ctypes.data_as(ctypes.c_void_p)))
        return out

    def eval_w(self, frac_idx, z) -> np.ndarray:
        """Complex discharge vector w_f(z) (andfn/hpc/hpc_fracture.py:139-175)."""
        frac_idx, z = points_args(frac_idx, z)
        out = np.empty(len(z), np.complex128)
        _ffi.check(_ffi.lib().andfn_b200_eval_w(self._h, frac_idx.ctypes.data_as(ctypes.c_void_p),
                                               z.ctypes.data_as(ctypes.c_void_p), len(z),
                                               out.ctypes.data_as(ctypes.c_void_p)))
        return out
