"""Record layouts of the reference's structured arrays.

AnDFN's solver works on two packed numpy record dtypes,
``element_dtype_hpc`` (andfn/element.py:45-69) and ``fracture_dtype_hpc``
(andfn/element.py:146-159), whose array fields are sized by the YAML-set
``MAX_NCOEF`` / ``MAX_ELEMENTS`` (andfn/element.py:13-20).  The drop-in must
read and write exactly these records, so the field names, order and types
below are the same as the reference's; ``layout_of`` turns any such dtype
into the byte-offset table the C ABI takes.
"""
from __future__ import annotations

import ctypes

import numpy as np

MAX_NCOEF_DEFAULT = 200
MAX_ELEMENTS_DEFAULT = 500

ELEMENT_TYPES = {0: "intersection", 1: "bounding_circle", 2: "well", 3: "constant_head_line",
                 4: "impermeable_circle", 5: "impermeable_line"}


def element_dtype(max_ncoef: int = MAX_NCOEF_DEFAULT) -> np.dtype:
    return np.dtype([
        ("_id", np.int_), ("_type", np.int_), ("frac0", np.int_), ("frac1", np.int_),
        ("endpoints0", np.complex128, 2), ("endpoints1", np.complex128, 2),
        ("radius", np.float64), ("center", np.complex128), ("head", np.float64),
        ("phi", np.float64), ("ncoef", np.int_), ("nint", np.int_), ("q", np.float64),
        ("thetas", np.float64, max_ncoef * 2), ("coef", np.complex128, max_ncoef),
        ("old_coef", np.complex128, max_ncoef), ("dpsi_corr", np.float64, max_ncoef * 2),
        ("error", np.float64), ("error_old", np.float64), ("error_old2", np.float64),
        ("error_coef", np.float64),
    ])


def fracture_dtype(max_elements: int = MAX_ELEMENTS_DEFAULT) -> np.dtype:
    return np.dtype([
        ("_id", np.int_), ("t", np.float64), ("radius", np.float64),
        ("center", np.float64, 3), ("normal", np.float64, 3), ("x_vector", np.float64, 3),
        ("y_vector", np.float64, 3), ("elements", np.int_, max_elements),
        ("nelements", np.int_), ("constant", np.float64),
    ])


# dtype_constants (andfn/constants.py:13-29)
constants_dtype = np.dtype([
    ("RHO", np.float64), ("G", np.float64), ("SE_FACTOR", np.float64),
    ("MAX_ITERATIONS", np.int32), ("MAX_ERROR", np.float64), ("MAX_NCOEF", np.int32),
    ("DAMPING", np.float64), ("COEF_INCREASE", np.int32), ("COEF_RATIO", np.float64),
    ("MAX_ELEMENTS", np.int32), ("NCOEF", np.int32), ("NINT", np.int32), ("NUM_THREADS", np.int32),
])


def default_constants(**overrides) -> np.ndarray:
    """The reference's defaults (andfn/constants.py:89-106) with overrides."""
    c = np.array((1000.0, 9.81, 0.9, 50, 1e-6, 150, 0.5, 5, 0.05, 150, 5, 10, -1), dtype=constants_dtype)
    for k, v in overrides.items():
        c[k] = v
    return c


class AndfnLayout(ctypes.Structure):
    """Mirror of ``AndfnLayout`` in include/andfn_b200.h."""

    _fields_ = [(n, ctypes.c_int64) for n in (
        "elem_size", "e_id", "e_type", "e_frac0", "e_frac1", "e_endpoints0",
        "e_endpoints1", "e_radius", "e_center", "e_head", "e_phi", "e_ncoef",
        "e_nint", "e_q", "e_thetas", "e_coef", "e_old_coef", "e_dpsi_corr",
        "e_error", "e_error_old", "e_error_old2", "e_error_coef", "max_ncoef",
        "frac_size", "f_id", "f_t", "f_radius", "f_center", "f_normal",
        "f_x_vector", "f_y_vector", "f_elements", "f_nelements", "f_constant",
        "max_elements")]


class AndfnConstants(ctypes.Structure):
    _fields_ = [("max_error", ctypes.c_double), ("max_iterations", ctypes.c_int64),
                ("max_ncoef", ctypes.c_int64), ("damping", ctypes.c_double),
                ("coef_increase", ctypes.c_int64), ("coef_ratio", ctypes.c_double)]


class AndfnSolveStats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int64), ("cnt_error", ctypes.c_int64), ("error", ctypes.c_double),
                ("error_coef", ctypes.c_double), ("error_q", ctypes.c_double),
                ("worst_element", ctypes.c_int64), ("n_unknowns", ctypes.c_int64),
                ("nnz_matrix", ctypes.c_int64), ("nnz_factors", ctypes.c_int64),
                ("gpu_launches", ctypes.c_int64), ("ms_upload", ctypes.c_double),
                ("ms_setup", ctypes.c_double), ("ms_factor", ctypes.c_double),
                ("ms_iterate", ctypes.c_double), ("ms_download", ctypes.c_double),
                ("ms_total", ctypes.c_double), ("status", ctypes.c_int32), ("device", ctypes.c_int32),
                ("h2d_bytes", ctypes.c_int64), ("d2h_bytes", ctypes.c_int64), ("dense_tail", ctypes.c_int64),
                ("levels_l", ctypes.c_int64), ("levels_u", ctypes.c_int64),
                ("ms_create_upload", ctypes.c_double), ("ms_create_tables", ctypes.c_double),
                ("ms_create_order", ctypes.c_double), ("tri_cycles", ctypes.c_int64 * 8),
                ("explicit_inverse", ctypes.c_int64), ("ms_factor_sparse", ctypes.c_double),
                ("ms_factor_dense", ctypes.c_double), ("ms_factor_levels", ctypes.c_double),
                ("ms_inverse", ctypes.c_double), ("refined_solves", ctypes.c_int64),
                ("sweep_variant", ctypes.c_int64), ("loop_launches", ctypes.c_int64), ("ms_alloc", ctypes.c_double),
                ("refine_f32", ctypes.c_int64)]

    def as_dict(self) -> dict:
        d = {name: getattr(self, name) for name, _ in self._fields_}
        d["tri_cycles"] = list(self.tri_cycles)
        return d

class AndfnAdjointStats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int64), ("residual", ctypes.c_double), ("lam_norm", ctypes.c_double),
                ("restart", ctypes.c_int64), ("ms_setup", ctypes.c_double), ("ms_iterate", ctypes.c_double),
                ("ms_total", ctypes.c_double), ("gpu_launches", ctypes.c_int64), ("status", ctypes.c_int32),
                ("pad", ctypes.c_int32)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "pad"}


class AndfnResidual(ctypes.Structure):
    _fields_ = [("bc_max", ctypes.c_double), ("bc_worst", ctypes.c_int64), ("flux_max", ctypes.c_double),
                ("flux_worst", ctypes.c_int64), ("h_scale", ctypes.c_double), ("q_scale", ctypes.c_double)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


_INT_FIELDS = ("_id", "_type", "frac0", "frac1", "ncoef", "nint")


def layout_of(elem_dtype: np.dtype, frac_dtype: np.dtype) -> AndfnLayout:
    """Byte offsets of every field the solver touches, from ``dtype.fields``."""
    ef, ff = elem_dtype.fields, frac_dtype.fields
    if ef is None or ff is None:
        raise TypeError("element/fracture arrays must be structured arrays")
    for name in _INT_FIELDS:
        if ef[name][0] != np.dtype(np.int64):
            raise TypeError(f"element field {name} must be int64")
    lay = AndfnLayout()
    lay.elem_size = elem_dtype.itemsize
    for name in ("_id", "_type", "frac0", "frac1", "endpoints0", "endpoints1", "radius", "center",
                 "head", "phi", "ncoef", "nint", "q", "thetas", "coef", "old_coef", "dpsi_corr",
                 "error", "error_old", "error_old2", "error_coef"):
        setattr(lay, "e_" + name.lstrip("_"), ef[name][1])
    lay.max_ncoef = ef["coef"][0].shape[0]
    lay.frac_size = frac_dtype.itemsize
    for name in ("_id", "t", "radius", "center", "normal", "x_vector", "y_vector", "elements",
                 "nelements", "constant"):
        setattr(lay, "f_" + name.lstrip("_"), ff[name][1])
    lay.max_elements = ff["elements"][0].shape[0]
    return lay


def constants_struct(constants) -> AndfnConstants:
    def g(k):
        v = constants[k]
        return v.item() if hasattr(v, "item") else v
    c = AndfnConstants()
    c.max_error = float(g("MAX_ERROR"))
    c.max_iterations = int(g("MAX_ITERATIONS"))
    c.max_ncoef = int(g("MAX_NCOEF"))
    c.damping = float(g("DAMPING"))
    c.coef_increase = int(g("COEF_INCREASE"))
    c.coef_ratio = float(g("COEF_RATIO"))
    return c
