"""Flow-field evaluations of a solved network on the GPU.

Mirrors the field functions of andfn/hpc/hpc_fracture.py with the same
arguments and results:

* ``sunflower_spiral(n_in, n_bnd)``                      hpc_fracture.py:20-49
* ``get_flow_nets(F, n_points, n_boundary_points, E)``   hpc_fracture.py:254-300
* ``get_heads(F, E, z_array)``                            hpc_fracture.py:303-343
* ``calc_w(F, E, frac_idx, z)``                           hpc_fracture.py:139-175 (vectorised over points)
* ``calc_velocity(F, E, frac_idx, z, aperture)``          andfn/fracture.py:481-497 (object-layer w)

The point evaluations run in the library (``andfn_b200_eval_omega``,
``andfn_b200_eval_heads``, ``andfn_b200_eval_w``): one GPU thread per point,
summing every element of the point's fracture.  ``solver`` may be an open
:class:`andfn_b200.Solver` whose device state is the solved network (then
nothing is uploaded); otherwise the records are uploaded for the call.
"""
from __future__ import annotations

import contextlib

import numpy as np

from .solver import Solver


def sunflower_spiral(n_in: int, n_bnd: int) -> np.ndarray:
    """n_in points of a golden-angle spiral in the unit disc (r = sqrt((i + 1/2) / n_in),
    theta = pi (1 + sqrt 5) (i + 1/2)) followed by n_bnd points exp(i theta) at
    linspace(0, 2 pi, n_bnd) on the unit circle."""
    idx = np.arange(0, n_in, dtype=np.float64) + 0.5
    r = np.sqrt(idx / n_in)
    theta = np.pi * (1 + 5 ** 0.5) * idx
    z = r * np.cos(theta) + 1j * r * np.sin(theta)
    return np.concatenate((z, np.exp(1j * np.linspace(0, 2 * np.pi, n_bnd))))


def map_2d_to_3d(fractures: np.ndarray, z: np.ndarray) -> np.ndarray:
    """3-D points Re z x_vector + Im z y_vector + center of every fracture
    (andfn/hpc/hpc_geometry_functions.py:103-132); z: [nf, n] -> [nf, n, 3]."""
    return (np.real(z)[:, :, None] * fractures["x_vector"][:, None, :]
            + np.imag(z)[:, :, None] * fractures["y_vector"][:, None, :]
            + fractures["center"][:, None, :])


@contextlib.contextmanager
def _handle(fractures, elements, solver, discharge_int):
    if solver is not None:
        yield solver
        return
    s = Solver(np.ascontiguousarray(fractures), np.ascontiguousarray(elements), discharge_int)
    try:
        yield s
    finally:
        s.close()


def _disc_points(fractures, z_unit):
    z = np.asarray(z_unit, np.complex128)[None, :] * fractures["radius"].astype(np.float64)[:, None]
    frac = np.repeat(np.arange(len(fractures), dtype=np.int64), z.shape[1])
    return z, frac


def get_flow_nets(fracture_struc_array, n_points, n_boundary_points, element_struc_array, *,
                  solver: Solver | None = None, discharge_int: int = 50):
    """Omega at the sunflower points of every fracture (scaled by its radius) and
    the points in 3-D.  Returns ``(flow_nets, pnts_3d)`` with the reference's
    shapes [nf, n, n] and [nf, n, 3], n = n_points + n_boundary_points; the
    reference fills every column of row i with Omega(z_i), so ``flow_nets`` is
    that broadcast as a read-only view of the [nf, n] values (no n^2 copy)."""
    F = fracture_struc_array
    n = int(n_points) + int(n_boundary_points)
    z, frac = _disc_points(F, sunflower_spiral(int(n_points), int(n_boundary_points)))
    with _handle(F, element_struc_array, solver, discharge_int) as s:
        om = s.eval_omega(frac, z.ravel()).reshape(len(F), n)
    return np.broadcast_to(om[:, :, None], (len(F), n, n)), map_2d_to_3d(F, z)


def get_heads(fracture_struc_array, element_struc_array, z_array, *, solver: Solver | None = None,
              discharge_int: int = 50):
    """Heads Re(Omega)/t at z_array (points of the unit disc, scaled by each
    fracture's radius) of every fracture, and the points in 3-D: ``(heads [nf, n],
    pnts_3d [nf, n, 3])``."""
    F = fracture_struc_array
    z, frac = _disc_points(F, z_array)
    with _handle(F, element_struc_array, solver, discharge_int) as s:
        h = s.eval_heads(frac, z.ravel()).reshape(z.shape)
    return h, map_2d_to_3d(F, z)


def calc_w(fracture_struc_array, element_struc_array, frac_idx, z, *, solver: Solver | None = None,
           discharge_int: int = 50) -> np.ndarray:
    """Complex discharge vector of fracture frac_idx[i] at z[i] (the reference's
    per-point ``calc_w(F[f], z, E)`` with exclude = -1)."""
    with _handle(fracture_struc_array, element_struc_array, solver, discharge_int) as s:
        return s.eval_w(np.atleast_1d(frac_idx), np.atleast_1d(z))


def calc_velocity(fracture_struc_array, element_struc_array, frac_idx, z, aperture, *,
                  solver: Solver | None = None, discharge_int: int = 50) -> np.ndarray:
    """Fracture.calc_velocity (andfn/fracture.py:481-497): |w| / aperture, with w
    the discharge vector of the reference's Fracture objects (Fracture.calc_w,
    andfn/fracture.py:453-478: bounding circles with -1/R and NaN outside, wells
    and impermeable circles NaN inside, impermeable elements included), which
    differs from the consolidated ``calc_w`` above.  The aperture is an attribute
    of the Fracture objects, not of the records, so it is passed in: a scalar or
    one value per point."""
    from .track import calc_w_object
    w = calc_w_object(fracture_struc_array, element_struc_array, frac_idx, z, solver=solver,
                      discharge_int=discharge_int)
    return np.abs(w) / np.asarray(aperture, np.float64)
