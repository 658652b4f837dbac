"""CPU oracle for the AnDFN analytic-element solve -- TEST INFRASTRUCTURE ONLY.

This module restates ``andfn.hpc.hpc_solve.solve`` (andfn/hpc/hpc_solve.py:55-257)
on top of ``oracle/andfn_oracle.c`` (a C restatement of the Numba kernels in
andfn/hpc/*.py).  Only the tests, ``__graft_entry__.smoke()`` and the CPU leg of
``bench.py`` use it, always as the checker or the timed CPU baseline; the
product package ``andfn_b200`` never imports it.

Third-party arithmetic on the path: the discharge system is factorised with
``scipy.sparse.linalg.splu`` (SuperLU, default COLAMD column ordering and
partial pivoting) exactly as the reference does at andfn/hpc/hpc_solve.py:121,651.
The installed SciPy version is recorded by ``scipy_version()``.

Pinning: tests/test_oracle_golden.py checks this oracle against golden vectors
produced by running the reference's own solver (tests/golden/make_golden.py).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")


class Layout(ctypes.Structure):
    """Mirror of AndfnLayout in include/andfn_b200.h."""

    _fields_ = [(n, ctypes.c_int64) for n in (
        "elem_size", "e_id", "e_type", "e_frac0", "e_frac1", "e_endpoints0",
        "e_endpoints1", "e_radius", "e_center", "e_head", "e_phi", "e_ncoef",
        "e_nint", "e_q", "e_thetas", "e_coef", "e_old_coef", "e_dpsi_corr",
        "e_error", "e_error_old", "e_error_old2", "e_error_coef", "max_ncoef",
        "frac_size", "f_id", "f_t", "f_radius", "f_center", "f_normal",
        "f_x_vector", "f_y_vector", "f_elements", "f_nelements", "f_constant",
        "max_elements")]


def layout_of(elem_dtype: np.dtype, frac_dtype: np.dtype) -> Layout:
    ef, ff = elem_dtype.fields, frac_dtype.fields
    lay = Layout()
    lay.elem_size = elem_dtype.itemsize
    for name in ("_id", "_type", "frac0", "frac1", "endpoints0", "endpoints1",
                 "radius", "center", "head", "phi", "ncoef", "nint", "q",
                 "thetas", "coef", "old_coef", "dpsi_corr", "error", "error_old",
                 "error_old2", "error_coef"):
        setattr(lay, "e_" + name.lstrip("_"), ef[name][1])
    lay.max_ncoef = ef["coef"][0].shape[0]
    lay.frac_size = frac_dtype.itemsize
    for name in ("_id", "t", "radius", "center", "normal", "x_vector",
                 "y_vector", "elements", "nelements", "constant"):
        setattr(lay, "f_" + name.lstrip("_"), ff[name][1])
    lay.max_elements = ff["elements"][0].shape[0]
    return lay


def build(force: bool = False) -> str:
    """Compile the C oracle with gcc (no FMA contraction, OpenMP)."""
    src = os.path.join(HERE, "andfn_oracle.c")
    if (not force and os.path.exists(LIB_PATH)
            and os.path.getmtime(LIB_PATH) >= os.path.getmtime(src)):
        return LIB_PATH
    os.makedirs(os.path.dirname(LIB_PATH), exist_ok=True)
    cmd = ["gcc", "-O2", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
           "-fno-fast-math", "-std=c11", "-o", LIB_PATH, src, "-lm"]
    subprocess.check_call(cmd)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = build()
        L = ctypes.CDLL(path)
        P, I64, D = ctypes.c_void_p, ctypes.c_int64, ctypes.c_double
        L.oracle_create.restype = P
        L.oracle_create.argtypes = [I64, I64, I64]
        L.oracle_destroy.argtypes = [P]
        L.oracle_num_threads.restype = ctypes.c_int
        L.oracle_set_num_threads.argtypes = [ctypes.c_int]
        L.oracle_init.argtypes = [P, P, P, I64]
        L.oracle_z_int.argtypes = [P, P, P, I64, I64, P, P]
        L.oracle_count_nnz.restype = I64
        L.oracle_count_nnz.argtypes = [P, P, P, I64, P, I64, P]
        L.oracle_fill_matrix.argtypes = [P, P, P, I64, P, I64, P, P, P, I64, P, P, P, P]
        L.oracle_head_vector.argtypes = [P, P, I64, P, I64, P, I64, P, P, I64, P]
        L.oracle_post_solve.argtypes = [P, P, P, I64, P, I64, P]
        L.oracle_element_solver.restype = ctypes.c_int
        L.oracle_element_solver.argtypes = [P, P, P, I64, P, I64, D]
        L.oracle_element_solver2.restype = ctypes.c_int
        L.oracle_element_solver2.argtypes = [P, P, P, I64, P, I64, D, I64, D, I64, I64, D]
        L.oracle_eval_omega.argtypes = [P, P, P, P, P, I64, P]
        L.oracle_eval_heads.argtypes = [P, P, P, P, P, I64, P]
        L.oracle_collocation_omega.argtypes = [P, P, P, P, I64, ctypes.c_int, P]
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def scipy_version() -> str:
    import scipy
    return scipy.__version__


def discharge_element_ids(elements: np.ndarray) -> np.ndarray:
    """hpc_solve.py:283-307: ids of types 0, 2, 3 in element order."""
    t = elements["_type"]
    return np.nonzero((t == 0) | (t == 2) | (t == 3))[0].astype(np.int64)


def specified_discharge_wells(elements: np.ndarray) -> np.ndarray:
    """Mask of the wells whose discharge is prescribed (an extension: the
    reference's wells prescribe a head, andfn/well.py:38, and their q is an
    unknown of the discharge system, hpc_solve.py:1451-1459).  Such a well is
    marked by a NaN head; its record's q is the prescribed discharge."""
    return (elements["_type"] == 2) & np.isnan(elements["head"])


class Oracle:
    """State of one oracle solve (the reference's work_array and tables)."""

    def __init__(self, fractures: np.ndarray, elements: np.ndarray, discharge_int: int):
        assert fractures.flags.c_contiguous and elements.flags.c_contiguous
        self.F, self.E = fractures, elements
        self.D = int(discharge_int)
        self.lay = layout_of(elements.dtype, fractures.dtype)
        self.L = lib()
        self.ne, self.nf = len(elements), len(fractures)
        self.ctx = self.L.oracle_create(self.ne, self.lay.max_ncoef, self.lay.max_elements)
        self.de = discharge_element_ids(elements)
        self.n_de = len(self.de)
        D = self.D
        self.z0 = np.zeros((max(self.n_de, 1), D), np.complex128)
        self.z1 = np.zeros((max(self.n_de, 1), D), np.complex128)
        self.L.oracle_z_int(ctypes.byref(self.lay), _ptr(self.E), _ptr(self.de), self.n_de, D,
                            _ptr(self.z0), _ptr(self.z1))

    def __del__(self):
        try:
            self.L.oracle_destroy(self.ctx)
        except Exception:
            pass

    # --- discharge system (hpc_solve.py:832-887, 1061-1201) ---------------
    def build_matrix(self):
        import scipy.sparse as sp
        size = self.n_de + self.nf
        nnz_per_row = np.zeros(size, np.int64)
        total = self.L.oracle_count_nnz(ctypes.byref(self.lay), _ptr(self.E), _ptr(self.F), self.nf,
                                        _ptr(self.de), self.n_de, _ptr(nnz_per_row))
        row_offsets = np.zeros(size, np.int64)
        row_offsets[1:] = np.cumsum(nnz_per_row)[:-1]
        rows = np.empty(total, np.int64)
        cols = np.empty(total, np.int64)
        data = np.empty(total, np.float64)
        id_to_pos = np.full(int(self.E["_id"].max()) + 1, -1, np.int64)
        id_to_pos[self.E["_id"][self.de]] = np.arange(self.n_de)
        self.L.oracle_fill_matrix(ctypes.byref(self.lay), _ptr(self.E), _ptr(self.F), self.nf, _ptr(self.de),
                                  self.n_de, _ptr(id_to_pos), _ptr(self.z0), _ptr(self.z1), self.D,
                                  _ptr(row_offsets), _ptr(rows), _ptr(cols), _ptr(data))
        return sp.csc_matrix((data, (rows, cols)), shape=(size, size))

    def init(self):
        self.L.oracle_init(self.ctx, ctypes.byref(self.lay), _ptr(self.E), self.ne)

    def head_vector(self) -> np.ndarray:
        head = np.zeros(self.n_de + self.nf)
        self.L.oracle_head_vector(ctypes.byref(self.lay), _ptr(self.E), self.ne, _ptr(self.F), self.nf,
                                  _ptr(self.de), self.n_de, _ptr(self.z0), _ptr(self.z1), self.D, _ptr(head))
        return head

    def post_solve(self, x: np.ndarray):
        self.L.oracle_post_solve(ctypes.byref(self.lay), _ptr(self.E), _ptr(self.F), self.nf, _ptr(self.de),
                                 self.n_de, _ptr(np.ascontiguousarray(x)))

    def element_solver(self, damping: float):
        rc = self.L.oracle_element_solver(self.ctx, ctypes.byref(self.lay), _ptr(self.E), self.ne,
                                          _ptr(self.F), self.nf, damping)
        if rc:
            raise RuntimeError("oracle element_solver failed (capacity exceeded)")

    def element_solver2(self, max_error, nit, coef_ratio, max_coef, coef_increase, damping):
        rc = self.L.oracle_element_solver2(self.ctx, ctypes.byref(self.lay), _ptr(self.E), self.ne,
                                           _ptr(self.F), self.nf, max_error, nit, coef_ratio, max_coef,
                                           coef_increase, damping)
        if rc:
            raise RuntimeError("oracle element_solver2 failed (capacity exceeded)")

    def collocation_omega(self, el: int, side: int) -> np.ndarray:
        out = np.zeros(int(self.E["nint"][el]), np.complex128)
        self.L.oracle_collocation_omega(self.ctx, ctypes.byref(self.lay), _ptr(self.E), _ptr(self.F), el,
                                        side, _ptr(out))
        return out


def _const(constants, name):
    return constants[name].item() if hasattr(constants[name], "item") else constants[name]


def solve(fracture_struc_array, element_struc_array, discharge_int, constants, ntype_elements=None,
          stats: dict | None = None, max_iterations: int | None = None, refine: bool = False):
    """Restatement of andfn/hpc/hpc_solve.py:55-257 (same in-place contract).

    ``constants`` is a dtype_constants record or a mapping with the keys
    MAX_ERROR, MAX_ITERATIONS, COEF_RATIO, MAX_NCOEF, COEF_INCREASE, DAMPING.

    ``refine=True`` (not the reference's algorithm; off by default) adds one
    step of iterative refinement to every discharge solve, x += LU^-1 (b - A x).
    The reference's unrefined SuperLU solves of an ill-conditioned system
    (condition ~1e12) carry round-off of ~1e-10 relative that changes with
    every right-hand side, so a quantity of the solved state is a smooth
    function of the inputs only down to that level; with the refinement it is
    smooth to ~1e-15, which finite-difference checks of derivatives need.
    """
    import scipy.sparse.linalg as spla

    max_error = float(_const(constants, "MAX_ERROR"))
    max_it = int(_const(constants, "MAX_ITERATIONS")) if max_iterations is None else int(max_iterations)
    coef_ratio = float(_const(constants, "COEF_RATIO"))
    max_coef = int(_const(constants, "MAX_NCOEF"))
    coef_increase = int(_const(constants, "COEF_INCREASE"))
    damping = float(_const(constants, "DAMPING"))

    F, E = fracture_struc_array, element_struc_array
    t_start = time.perf_counter()
    o = Oracle(F, E, discharge_int)
    size = o.n_de + o.nf
    # get_old_discharges (hpc_solve.py:765-775)
    discharges = np.zeros(o.n_de + int(E["frac0"].max()) + 1)
    discharges[: o.n_de] = E["q"][o.de]
    discharges[o.n_de: o.n_de + o.nf] = F["constant"]
    discharges = discharges[:size] if len(discharges) >= size else np.pad(discharges, (0, size - len(discharges)))
    A = o.build_matrix()
    # Wells with a prescribed discharge (specified_discharge_wells): their
    # rows and columns leave the system, and their known discharge moves to
    # the right-hand side of the other rows (the matrix entry times q, and
    # the well's +q in its fracture's continuity row).
    spec = np.zeros(size, bool)
    spec[: o.n_de] = specified_discharge_wells(E)[o.de]
    keep = ~spec
    q_spec = E["q"][o.de[spec[: o.n_de]]].copy()
    b_known = None
    if spec.any():
        A = A.tocsr()
        b_known = -(A[keep][:, np.nonzero(spec)[0]] @ q_spec)
        A = A[keep][:, keep].tocsc()
        discharges = discharges[keep]
    discharges_old = np.zeros(len(discharges))

    def scatter(x):
        if b_known is None:
            return x
        full = np.zeros(size)
        full[keep] = x
        full[spec] = q_spec
        return full

    t_mat = time.perf_counter()
    lu = spla.splu(A)
    t_lu = time.perf_counter()
    o.init()

    error = 1.0
    error_coef = 1.0
    nit = 0
    cnt_error = 0
    error_q = 1.0
    t_q = t_e = 0.0
    _id = 0
    while cnt_error < 2 and nit < max_it:
        nit += 1
        t0 = time.perf_counter()
        if error_q > max_error / 1e30:
            discharges_old[:] = discharges[:]
            head = o.head_vector()
            if b_known is not None:
                head = head[keep] + b_known
            discharges[:] = lu.solve(head)
            if refine:
                discharges += lu.solve(head - A @ discharges)
            o.post_solve(scatter(discharges))
            error_q = np.max(np.abs(discharges - discharges_old) / (np.max(np.abs(discharges_old)) + 1e-16))
        t1 = time.perf_counter()
        o.element_solver2(max_error, nit, coef_ratio, max_coef, coef_increase, damping)
        t2 = time.perf_counter()
        t_q += t1 - t0
        t_e += t2 - t1
        error = float(np.max(E["error"]))
        _id = int(np.argmax(E["error"]))
        error_coef = float(np.max(E["error_coef"]))
        if nit == max_it:
            o.element_solver(damping)
        if error_coef < max_error and error_q < max_error:
            cnt_error += 1
            error_q = 1e30
    if stats is not None:
        stats.update(dict(iterations=nit, cnt_error=cnt_error, error=error, error_coef=error_coef,
                          error_q=float(error_q), worst_element=_id, n_unknowns=A.shape[0], nnz_matrix=A.nnz,
                          nnz_factors=int(lu.L.nnz + lu.U.nnz), s_matrix=t_mat - t_start, s_lu=t_lu - t_mat,
                          s_discharge=t_q, s_elements=t_e, s_total=time.perf_counter() - t_start,
                          threads=lib().oracle_num_threads()))
    return element_struc_array


def eval_heads(fractures, elements, frac_idx, z) -> np.ndarray:
    """Heads Re(Omega_f(z))/t_f (andfn/hpc/hpc_fracture.py:205-252)."""
    lay = layout_of(elements.dtype, fractures.dtype)
    frac_idx = np.ascontiguousarray(frac_idx, np.int64)
    z = np.ascontiguousarray(z, np.complex128)
    out = np.zeros(len(z))
    lib().oracle_eval_heads(ctypes.byref(lay), _ptr(elements), _ptr(fractures), _ptr(frac_idx), _ptr(z),
                            len(z), _ptr(out))
    return out


def eval_omega(fractures, elements, frac_idx, z) -> np.ndarray:
    """Omega_f(z) (andfn/hpc/hpc_fracture.py:52-94, exclude = -1)."""
    lay = layout_of(elements.dtype, fractures.dtype)
    frac_idx = np.ascontiguousarray(frac_idx, np.int64)
    z = np.ascontiguousarray(z, np.complex128)
    out = np.zeros(len(z), np.complex128)
    lib().oracle_eval_omega(ctypes.byref(lay), _ptr(elements), _ptr(fractures), _ptr(frac_idx), _ptr(z),
                            len(z), _ptr(out))
    return out


def set_num_threads(n: int):
    lib().oracle_set_num_threads(int(n))


def num_threads() -> int:
    return int(lib().oracle_num_threads())


if __name__ == "__main__":
    print(build(force=True))
    print("threads", num_threads(), "scipy", scipy_version(), "pid", os.getpid())


# --- boundary-condition residual and flux balance (test/report restatement) ---
def collocation_points(elements, e, side=0):
    """The element's collocation points: z = map_chi_to_z(exp(i theta_k))
    (andfn/hpc/hpc_math_functions.py:279-284, 674-699)."""
    E = elements
    ty, n = int(E["_type"][e]), int(E["nint"][e])
    k = np.arange(n)
    th = 2 * np.pi * k / n if ty == 1 else (k + 0.5) * np.pi / n
    chi = np.exp(1j * th)
    if ty in (1, 4):
        return E["radius"][e] * chi + E["center"][e]
    ep = E["endpoints1"][e] if side else E["endpoints0"][e]
    a, b = ep[0], ep[1]
    return 0.5 * (0.5 * (chi + 1 / chi) * (b - a) + a + b)


def bc_residual(fractures, elements):
    """Per-element boundary-condition residual and per-fracture flux balance
    of a solved state, as andfn_b200_bc_residual defines them (the flux
    balance is Fracture.check_discharge, andfn/fracture.py:377-394)."""
    F, E = fractures, elements
    ty = E["_type"]
    t = F["t"]
    heads = np.abs(E["phi"] / t[E["frac0"]])[np.isin(ty, (2, 3))]
    hs = heads.max() if len(heads) and heads.max() > 0 else 1.0
    ne = len(E)
    res = np.zeros(ne)
    disch = np.isin(ty, (0, 2, 3))
    flux = np.zeros(len(F))
    ftot = np.zeros(len(F))
    for f in range(len(F)):
        els = F["elements"][f, : F["nelements"][f]]
        s = tot = 0.0
        for el in els:
            if not disch[el]:
                continue
            s += -E["q"][el] if (ty[el] == 0 and E["frac1"][el] == f) else E["q"][el]
            tot += abs(E["q"][el])
        flux[f] = abs(s)
        ftot[f] = tot
    qs = ftot.max() if len(ftot) and ftot.max() > 0 else 1.0
    for e in range(ne):
        f0 = int(E["frac0"][e])
        if ty[e] in (0, 3):
            z0 = collocation_points(E, e, 0)
            h0 = eval_omega(F, E, np.full(len(z0), f0), z0).real / t[f0]
            if ty[e] == 0:
                f1 = int(E["frac1"][e])
                z1 = collocation_points(E, e, 1)
                h1 = eval_omega(F, E, np.full(len(z1), f1), z1).real / t[f1]
                d = h0 - h1
            else:
                d = h0 - E["phi"][e] / t[f0]
            res[e] = np.abs(d).max() / hs if len(d) else 0.0
        elif ty[e] == 2:
            z = E["center"][e] + E["radius"][e] * np.exp(2j * np.pi * np.arange(16) / 16)
            h = eval_omega(F, E, np.full(16, f0), z).real / t[f0]
            res[e] = np.abs(h - E["phi"][e] / t[f0]).max() / hs
        else:
            z = collocation_points(E, e, 0)
            n = len(z)
            psi = eval_omega(F, E, np.full(n, f0), z).imag
            corr = np.concatenate([[0.0], np.cumsum(E["dpsi_corr"][e][: n - 1])])
            psi = psi - corr
            res[e] = (psi.max() - psi.min()) / qs
    return {"elem": res, "flux": flux, "h_scale": hs, "q_scale": qs, "bc_max": float(res.max()),
            "flux_max": float(flux.max() / qs)}


# ---------------------------------------------------------------------------
# Flow-field evaluations (test infrastructure: restatements the GPU results
# are checked against; pure Python, small cases).
# ---------------------------------------------------------------------------
def sunflower_spiral(n_in: int, n_bnd: int) -> np.ndarray:
    """Unit-disc sample points (andfn/hpc/hpc_fracture.py:20-49): n_in points on
    a golden-angle spiral, r = sqrt((i + 1/2) / n_in), theta = pi (1 + sqrt 5)
    (i + 1/2), then n_bnd points exp(i theta) at linspace(0, 2 pi, n_bnd)."""
    idx = np.arange(0, n_in, dtype=np.float64) + 0.5
    r = np.sqrt(idx / n_in)
    th = np.pi * (1 + 5 ** 0.5) * idx
    z = r * np.cos(th) + 1j * r * np.sin(th)
    return np.concatenate((z, np.exp(1j * np.linspace(0, 2 * np.pi, n_bnd))))


def _line_chi(z, ep):
    # andfn/hpc/hpc_geometry_functions.py:12-31
    big_z = (2 * z - ep[0] - ep[1]) / (ep[1] - ep[0])
    return big_z + np.sqrt(big_z - 1) * np.sqrt(big_z + 1)


def _asym_d1(chi, coef):
    # andfn/hpc/hpc_math_functions.py:76-100: d/dchi sum_k c_k chi^-k
    res = 0j
    n = len(coef)
    for k in range(n):
        res -= coef[n - k - 1] * (n - k - 1)
        res /= chi
    return res


def _taylor_d1(chi, coef):
    # andfn/hpc/hpc_math_functions.py:164-190: d/dchi sum_k c_k chi^k
    res = 0j
    n = len(coef)
    for k in range(n - 2):
        res += coef[n - k - 1] * (n - k - 1)
        res *= chi
    return res + coef[1]


def calc_w(fractures, elements, f: int, z: complex) -> complex:
    """Complex discharge vector of fracture f at z (andfn/hpc/hpc_fracture.py:139-175):
    the sum over its intersections (hpc_intersection.py:179-225, the second
    fracture's side with -coef, +q/(2 pi chi) and its own endpoints), bounding
    circle (hpc_bounding_circle.py:97-115: derivative of the Taylor series in
    chi = z / R, no chain-rule factor, center ignored), wells (hpc_well.py:89-108)
    and constant-head lines (hpc_const_head_line.py:135-164); impermeable
    elements do not contribute."""
    fr = fractures[f]
    w = 0j
    for k in range(int(fr["nelements"])):
        el = elements[int(fr["elements"][k])]
        t = int(el["_type"])
        if t == 0 or t == 3:
            side1 = t == 0 and int(fr["_id"]) != int(el["frac0"])
            ep = el["endpoints1"] if side1 else el["endpoints0"]
            chi = complex(_line_chi(complex(z), ep))
            c = el["coef"][: int(el["ncoef"])]
            if side1:
                ww = -_asym_d1(chi, -c) + el["q"] / (2 * np.pi * chi)
            else:
                ww = -_asym_d1(chi, c) - el["q"] / (2 * np.pi * chi)
            ww *= 2 * chi ** 2 / (chi ** 2 - 1) * 2 / (ep[1] - ep[0])
        elif t == 1:
            chi = complex(z) / el["radius"]
            ww = _taylor_d1(chi, el["coef"][: int(el["ncoef"])])
        elif t == 2:
            chi = (complex(z) - el["center"]) / el["radius"]
            ww = -el["q"] / (2 * np.pi * chi) / el["radius"]
        else:
            continue
        w += ww
    return complex(w)
