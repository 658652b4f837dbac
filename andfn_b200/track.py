"""Streamline (particle) tracking on the GPU.

Mirrors the tracking functions of the reference's DFN class on the records of
a solved network:

* ``streamline_tracking(F, E, z0, frac, elevation, ds, max_length, backward, aperture)``
                                      DFN.streamline_tracking, andfn/dfn.py:2643-2722
* ``streamlines(F, E, z0, frac, ds, max_length, elevation, remove_false, backward, aperture)``
                                      the tracing of DFN.plot_streamline_tracking,
                                      andfn/dfn.py:2558-2641, without the plotter: every
                                      start point with every elevation, then the 3-D lines
* ``get_travel_time_and_length(streamline, velocity)``
                                      DFN.get_travel_time_and_length, andfn/dfn.py:2848-2903

All particles are traced by one kernel launch (``andfn_b200_track``): a group
of 8 GPU lanes per particle, which share each sum over the fracture's elements,
follows its streamline through every fracture it enters.  The field is the object layer's Fracture.calc_w (andfn/fracture.py:
453-478), which differs from the consolidated calc_w of andfn.hpc at bounding
circles and impermeable elements; ``calc_w_object`` evaluates it at points.
Fracture apertures belong to the reference's Fracture objects, not to the
records, so they are passed in (a scalar or one value per fracture).

Elements are referred to by record index; -1 stands for the reference's False.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _ffi
from .fracture import _handle, map_2d_to_3d
from .solver import Solver, points_args

TRACK_DONE, TRACK_TRUNCATED = 0, 1


@dataclass
class Traces:
    """Raw result of one tracking launch: ``cap`` slots per particle."""
    z: np.ndarray          # complex128 [npart, cap]
    velocity: np.ndarray   # float64 [npart, cap]
    segment: np.ndarray    # int64 [npart, cap] segment index of each point
    fracture: np.ndarray   # int64 [npart, cap] fracture of each point
    npoints: np.ndarray    # int64 [npart]
    element: np.ndarray    # int64 [npart] last element, -1 = none
    status: np.ndarray     # int32 [npart] TRACK_DONE / TRACK_TRUNCATED

    def trace(self, i: int):
        """Particle i in the reference's return form: (list of segment point
        arrays, list of segment fractures, list of segment velocity arrays,
        last element or -1)."""
        n = int(self.npoints[i])
        z, v, seg, fr = self.z[i, :n], self.velocity[i, :n], self.segment[i, :n], self.fracture[i, :n]
        cuts = np.flatnonzero(np.diff(seg)) + 1
        starts = np.concatenate(([0], cuts)) if n else np.zeros(0, np.int64)
        ends = np.concatenate((cuts, [n])) if n else np.zeros(0, np.int64)
        return ([z[a:b].copy() for a, b in zip(starts, ends)], [int(fr[a]) for a in starts],
                [v[a:b].copy() for a, b in zip(starts, ends)], int(self.element[i]))


def _aperture(fractures, aperture) -> np.ndarray:
    if aperture is None:
        raise ValueError("fracture apertures are needed for velocities (Fracture.aperture)")
    a = np.broadcast_to(np.asarray(aperture, np.float64), (len(fractures),))
    return np.ascontiguousarray(a)


def track(solver: Solver, aperture, frac, z0, elevation=0.0, ds: float = 1e-2, max_length: int = 1000,
          backward=False, cap: int | None = None) -> Traces:
    """Trace every particle (frac[i], z0[i], elevation[i]) on the solved network
    of ``solver`` in one launch.  ``cap`` slots per particle default to
    max_length + 66; a trace that needs more stops with TRACK_TRUNCATED."""
    F = solver.fractures
    ap = _aperture(F, aperture)
    z0 = np.ascontiguousarray(np.atleast_1d(z0), np.complex128)
    n = len(z0)
    frac = np.ascontiguousarray(np.broadcast_to(np.asarray(frac, np.int64), (n,)))
    elev = np.ascontiguousarray(np.broadcast_to(np.asarray(elevation, np.float64), (n,)))
    cap = int(max_length) + 66 if cap is None else int(cap)
    out = Traces(np.zeros((n, cap), np.complex128), np.zeros((n, cap)), np.zeros((n, cap), np.int64),
                 np.zeros((n, cap), np.int64), np.zeros(n, np.int64), np.zeros(n, np.int64), np.zeros(n, np.int32))
    P = ctypes.c_void_p
    _ffi.check(_ffi.lib().andfn_b200_track(
        solver._h, F.ctypes.data_as(P), len(F), ap.ctypes.data_as(P), n, frac.ctypes.data_as(P),
        z0.ctypes.data_as(P), elev.ctypes.data_as(P), float(ds), int(max_length), int(bool(backward)), cap,
        out.z.ctypes.data_as(P), out.velocity.ctypes.data_as(P), out.segment.ctypes.data_as(P),
        out.fracture.ctypes.data_as(P), out.npoints.ctypes.data_as(P), out.element.ctypes.data_as(P),
        out.status.ctypes.data_as(P)))
    return out


def calc_w_object(fracture_struc_array, element_struc_array, frac_idx, z, *, solver: Solver | None = None,
                  discharge_int: int = 50) -> np.ndarray:
    """Fracture.calc_w of the object layer (andfn/fracture.py:453-478) at points."""
    frac_idx, z = points_args(np.atleast_1d(frac_idx), np.atleast_1d(z))
    out = np.empty(len(z), np.complex128)
    P = ctypes.c_void_p
    with _handle(fracture_struc_array, element_struc_array, solver, discharge_int) as s:
        _ffi.check(_ffi.lib().andfn_b200_eval_w_object(s._h, frac_idx.ctypes.data_as(P), z.ctypes.data_as(P),
                                                      len(z), out.ctypes.data_as(P)))
    return out


def streamline_tracking(fracture_struc_array, element_struc_array, z0, frac, elevation, ds, max_length,
                        backward=False, *, aperture, solver: Solver | None = None, discharge_int: int = 50):
    """One streamline (DFN.streamline_tracking): (segments, segment fractures,
    segment velocities, last element or -1)."""
    with _handle(fracture_struc_array, element_struc_array, solver, discharge_int) as s:
        return track(s, aperture, [frac], [z0], [elevation], ds, max_length, backward).trace(0)


def streamlines(fracture_struc_array, element_struc_array, z0, frac, ds=1e-2, max_length=1000, elevation=0.0,
                remove_false=True, backward=False, *, aperture, solver: Solver | None = None,
                discharge_int: int = 50):
    """The tracing of DFN.plot_streamline_tracking: every start point z0 on
    fracture ``frac`` with every elevation, all in one launch.  Returns the
    reference's four lists (streamlines, their fractures, velocities, last
    elements) and the 3-D polyline of each kept trace (traces with no points,
    and with remove_false those that end on no element, are left out)."""
    z0 = np.atleast_1d(np.asarray(z0, np.complex128))
    elevation = np.atleast_1d(np.asarray(elevation, np.float64))
    zz = np.repeat(z0, len(elevation))
    ee = np.tile(elevation, len(z0))
    with _handle(fracture_struc_array, element_struc_array, solver, discharge_int) as s:
        tr = track(s, aperture, frac, zz, ee, ds, max_length, backward)
    F = fracture_struc_array
    lines, fracs, vels, elems, lines_3d = [], [], [], [], []
    for i in range(len(zz)):
        seg, sf, v, e = tr.trace(i)
        lines.append(seg)
        fracs.append(sf)
        vels.append(v)
        elems.append(e)
        if not seg or (e < 0 and remove_false):
            continue
        lines_3d.append(np.concatenate([map_2d_to_3d(F[[f]], s_[None, :])[0] for s_, f in zip(seg, sf)]))
    return lines, fracs, vels, elems, lines_3d


def get_travel_time_and_length(streamline, velocity):
    """Travel time sum |dz| / v (velocity at the start of each step) and length
    sum |dz| over the segments, NaN points removed (andfn/dfn.py:2848-2903)."""
    time = 0.0
    length = 0.0
    for s, v in zip(streamline, velocity):
        s = np.asarray(s)
        v = np.asarray(v)
        mask = ~np.isnan(s) & ~np.isnan(v)
        s, v = s[mask], v[mask]
        time += np.sum(np.abs(s[1:] - s[:-1]) / v[:-1])
        length += np.sum(np.abs(s[1:] - s[:-1]))
    return time, length
