"""CPU oracle for streamline (particle) tracking -- TEST INFRASTRUCTURE ONLY.

Restates, on the consolidated records (fracture_dtype_hpc / element_dtype_hpc)
of a solved network, the object-layer tracking of the reference:

* ``calc_w_obj``            Fracture.calc_w (andfn/fracture.py:453-478) with the
                            element methods of the object layer (intersection.py:158-199,
                            const_head.py:166-185, bounding.py:49-108, well.py:129-153,
                            impermeable_object.py:131-156, 205-224);
* ``runge_kutta``           DFN.runge_kutta (andfn/dfn.py:2797-2846);
* ``check_streamline_exit`` DFN.check_streamline_exit (andfn/dfn.py:2724-2741) with the
                            crossing tests intersection.py:227-271, const_head.py:208-246,
                            well.py:162-200;
* ``get_exit_intersection`` DFN.get_exit_intersection (andfn/dfn.py:2743-2795);
* ``streamline_tracking``   DFN.streamline_tracking (andfn/dfn.py:2643-2722);
* ``travel_time_and_length`` DFN.get_travel_time_and_length (andfn/dfn.py:2848-2893).

The object layer's discharge vector differs from the consolidated one of
andfn/hpc/hpc_fracture.py:139-175: bounding circles carry the chain-rule
factor 1/R and a minus sign and give NaN outside |z/R| > 1 + 1e-5, wells and
impermeable circles give NaN inside, and impermeable elements contribute.

Fracture apertures are attributes of the reference's Fracture objects, not of
the records; they are passed as an array.  Elements are referred to by their
record index; ``-1`` stands for the reference's ``False`` (no element).

Pinning: tests/test_track_golden.py checks this module against traces of the
reference's own DFN.streamline_tracking (tests/golden/make_track_golden.py).
"""
from __future__ import annotations

import math

import numpy as np

ATOL_LINE = 1e-12   # intersection.py:227, const_head.py:208
ATOL_WELL = 1e-10   # well.py:162


def _csqrt(z: complex) -> complex:
    """Principal square root in the form Numba compiles for complex scalars
    (Algorithm 312, CACM 10 (1967), the NumPy npy_csqrt form), finite inputs."""
    a, b = z.real, z.imag
    if a == 0.0 and b == 0.0:
        return complex(abs(b), b)
    if a >= 0:
        t = math.sqrt((a + math.hypot(a, b)) * 0.5)
        return complex(t, b / (2 * t))
    t = math.sqrt((-a + math.hypot(a, b)) * 0.5)
    return complex(abs(b) / (2 * t), math.copysign(t, b))


def _line_chi(z, ep):
    """andfn/hpc/hpc_geometry_functions.py:12-31, which the object layer calls
    for scalars (andfn/geometry_functions.py:24-54).  It is compiled by Numba:
    complex division is CPython's Smith quotient (Python complex division is the
    same) and the square root is ``_csqrt``; with them a point exactly on the
    line falls on the same side of the branch cut as in the reference."""
    a, b, zz = complex(ep[0]), complex(ep[1]), complex(z)
    big_z = (2 * zz - a - b) / (b - a)
    if not (math.isfinite(big_z.real) and math.isfinite(big_z.imag)):
        return complex(np.sqrt(np.complex128(big_z - 1)) * np.sqrt(np.complex128(big_z + 1)) + big_z)
    return big_z + _csqrt(big_z - 1) * _csqrt(big_z + 1)


def _chi_to_z_line(chi, ep):
    # andfn/geometry_functions.py:57-82
    big_z = 1 / 2 * (chi + 1 / chi)
    return 1 / 2 * (big_z * (ep[1] - ep[0]) + ep[0] + ep[1])


def _asym_d1(chi, coef):
    # andfn/hpc/hpc_math_functions.py:76-100
    res = 0j
    n = len(coef)
    for k in range(n):
        res -= coef[n - k - 1] * (n - k - 1)
        res /= chi
    return res


def _taylor_d1(chi, coef):
    # andfn/hpc/hpc_math_functions.py:164-190
    res = 0j
    n = len(coef)
    for k in range(n - 2):
        res += coef[n - k - 1] * (n - k - 1)
        res *= chi
    return res + coef[1]


def _nan():
    return np.complex128(np.nan + 1j * np.nan)


def element_w(fractures, elements, f: int, e: int, z):
    """The object-layer calc_w of element e seen from fracture f."""
    el = elements[e]
    t = int(el["_type"])
    c = el["coef"][: int(el["ncoef"])]
    z = np.complex128(z)
    if t == 0 or t == 3:
        # intersection.py:174-199 (frac1 side: -coef, +q, endpoints1); const_head.py:180-185
        side1 = t == 0 and f != int(el["frac0"])
        ep = el["endpoints1"] if side1 else el["endpoints0"]
        chi = _line_chi(z, ep)
        if side1:
            w = -_asym_d1(chi, -c) + el["q"] / (2 * np.pi * chi)
        else:
            w = -_asym_d1(chi, c) - el["q"] / (2 * np.pi * chi)
        w *= 2 * chi ** 2 / (chi ** 2 - 1) * 2 / (ep[1] - ep[0])
        return w
    if t == 1:
        # bounding.py:49-71, 91-108: chi = z / R, NaN outside, -d/dchi Taylor / R
        chi = z / el["radius"]
        if np.abs(chi) > 1.0 + 1e-5:
            chi = _nan()
        w = -_taylor_d1(chi, c)
        w /= el["radius"]
        return w
    if t == 2:
        # well.py:144-153
        chi = (z - el["center"]) / el["radius"]
        if np.abs(chi) < 1.0 - 1e-10:
            return _nan()
        w = -el["q"] / (2 * np.pi * chi)
        w /= el["radius"]
        return w
    if t == 4:
        # impermeable_object.py:146-156
        chi = (z - el["center"]) / el["radius"]
        if np.abs(chi) < 1.0 - 1e-10:
            return _nan()
        w = -_asym_d1(chi, c)
        w /= el["radius"]
        return w
    # t == 5, impermeable_object.py:220-224
    ep = el["endpoints0"]
    chi = _line_chi(z, ep)
    w = -_asym_d1(chi, c)
    w *= 2 * chi ** 2 / (chi ** 2 - 1) * 2 / (ep[1] - ep[0])
    return w


def calc_w_obj(fractures, elements, f: int, z):
    """Fracture.calc_w (andfn/fracture.py:453-478): the sum over every element
    of fracture f in its element order."""
    fr = fractures[f]
    w = 0.0 + 0.0j
    for k in range(int(fr["nelements"])):
        w += element_w(fractures, elements, f, int(fr["elements"][k]), z)
    return w


def calc_velocity(fractures, elements, aperture, f: int, z):
    # andfn/fracture.py:481-497
    return np.abs(calc_w_obj(fractures, elements, f, z)) / aperture[f]


def map_2d_to_3d(fractures, f: int, z):
    # andfn/geometry_functions.py:161-190 (scalar form)
    fr = fractures[f]
    return np.real(z) * fr["x_vector"] + np.imag(z) * fr["y_vector"] + fr["center"]


def map_3d_to_2d(fractures, f: int, p):
    # andfn/geometry_functions.py:193-220
    fr = fractures[f]
    x = np.dot((p - fr["center"]), fr["x_vector"])
    y = np.dot((p - fr["center"]), fr["y_vector"])
    return x + 1j * y


def runge_kutta(fractures, elements, z0, f: int, ds, backward, tolerance=1e-6, max_it=10):
    """andfn/dfn.py:2797-2846: a unit step along conj(w) and up to max_it
    trapezoidal corrections; points beyond the fracture radius are pulled back
    inside."""
    radius = fractures[f]["radius"]
    if backward:
        ds = -ds
    w0 = calc_w_obj(fractures, elements, f, z0)
    if np.isnan(np.real(w0)):
        return np.nan + np.nan * 1j
    z1 = z0 + np.conj(w0) / np.abs(w0) * ds
    if np.abs(z1) > radius:
        z1 *= radius / (np.abs(z1) * (1 + 1e-5))
    dz = 1e99
    it = 0
    while dz > tolerance and it < max_it:
        w1 = calc_w_obj(fractures, elements, f, z1)
        if np.isnan(np.real(w1)):
            break
        z2 = z0 + np.conj(w0 + w1) / np.abs(w0 + w1) * ds
        if np.abs(z2) > radius:
            z2 *= radius / (np.abs(z2) * (1 + 1e-5))
        dz = np.abs(z2 - z1)
        z1 = z2
        it += 1
    return z1


def line_line_intersection(z0, z1, z2, z3):
    # andfn/geometry_functions.py:405-438
    determinant = (np.conj(z1) - np.conj(z0)) * (z3 - z2) - (z1 - z0) * (np.conj(z3) - np.conj(z2))
    if determinant == 0:
        return None
    z = (np.conj(z1) * z0 - z1 * np.conj(z0)) * (z3 - z2) - (z1 - z0) * ((np.conj(z3)) * z2 - z3 * np.conj(z2))
    z /= determinant
    return z


def line_circle_intersection(z0, z1, radius):
    # andfn/geometry_functions.py:359-402
    dx = np.real(z1 - z0)
    dy = np.imag(z1 - z0)
    if dx == 0:
        x = np.real(z0)
        with np.errstate(invalid="ignore"):
            y1 = np.sqrt(radius ** 2 - x ** 2)
        y2 = -y1
        return x + 1j * y1, x + 1j * y2
    m = dy / dx
    x0 = np.imag(z0) - m * np.real(z0)
    a = 1 + m ** 2
    b = 2 * x0 * m
    c = x0 ** 2 - radius ** 2
    discriminant = b ** 2 - 4 * a * c
    if discriminant < 0:
        return None, None
    sq = np.sqrt(discriminant)
    x1 = (-b + sq) / (2 * a)
    x2 = (-b - sq) / (2 * a)
    y1 = m * x1 + x0
    y2 = m * x2 + x0
    return x1 + 1j * y1, x2 + 1j * y2


def _line_crossing(z0, z1, ep, atol=ATOL_LINE):
    # intersection.py:247-271, const_head.py:226-246
    z = line_line_intersection(z0, z1, ep[0], ep[1])
    if z is None:
        return None
    if np.abs(np.abs(z - z0) + np.abs(z1 - z) - np.abs(z0 - z1)) > atol:
        return None
    if np.abs(np.abs(z - ep[0]) + np.abs(z - ep[1]) - np.abs(ep[0] - ep[1])) > atol:
        return None
    return z


def _well_crossing(z0, z1, el, atol=ATOL_WELL):
    # well.py:180-200
    chi0 = (z0 - el["center"]) / el["radius"]
    chi1 = (z1 - el["center"]) / el["radius"]
    chi2, chi3 = line_circle_intersection(chi0, chi1, 1.0)
    if chi2 is None:
        return None
    diff0 = np.abs(np.abs(chi2 - chi0) + np.abs(chi2 - chi1) - np.abs(chi1 - chi0))
    diff1 = np.abs(np.abs(chi3 - chi0) + np.abs(chi3 - chi1) - np.abs(chi1 - chi0))
    if diff0 > atol and diff1 > atol:
        return None
    chi2 *= 1 + atol
    chi3 *= 1 + atol
    z2 = chi2 * el["radius"] + el["center"]
    z3 = chi3 * el["radius"] + el["center"]
    if np.abs(z2 - z0) < np.abs(z3 - z0):
        return z2
    return z3


def check_streamline_exit(fractures, elements, z0, z1, f: int):
    """andfn/dfn.py:2724-2741: the first discharge element of fracture f (in its
    element order) whose boundary the segment z0 -> z1 crosses, and the
    crossing point; (None, -1) when there is none."""
    fr = fractures[f]
    for k in range(int(fr["nelements"])):
        e = int(fr["elements"][k])
        el = elements[e]
        t = int(el["_type"])
        if t == 0:
            ep = el["endpoints0"] if f == int(el["frac0"]) else el["endpoints1"]
            z2 = _line_crossing(z0, z1, ep)
        elif t == 3:
            z2 = _line_crossing(z0, z1, el["endpoints0"])
        elif t == 2:
            z2 = _well_crossing(z0, z1, el)
        else:
            continue
        if z2 is not None:
            return z2, e
    return None, -1


def get_exit_intersection(fractures, elements, z3d, e: int, f: int, f_old: int, elevation, dchi=1e-4):
    """andfn/dfn.py:2743-2795: the two points just off intersection e on either
    side in the new fracture f, the split of the incoming flow by |w| on the
    two sides, and the side (and rescaled elevation) the particle takes."""
    el = elements[e]
    endpoints = el["endpoints0"] if f == int(el["frac0"]) else el["endpoints1"]
    z = map_3d_to_2d(fractures, f, z3d)
    chi0 = _line_chi(z, endpoints)
    chi1 = np.conj(chi0)
    z0 = _chi_to_z_line(chi0 * (1 + dchi), endpoints)
    z1 = _chi_to_z_line(chi1 * (1 + dchi), endpoints)
    w0 = calc_w_obj(fractures, elements, f, z0)
    w1 = calc_w_obj(fractures, elements, f, z1)
    abs_w0 = np.abs(w0)
    abs_w1 = np.abs(w1)
    divide = abs_w0 / (abs_w0 + abs_w1)
    pointz0 = map_2d_to_3d(fractures, f, z0)
    nz0 = np.dot((pointz0 - z3d), fractures[f_old]["normal"])
    if nz0 < 0:
        up, down = z1, z0
    else:
        up, down = z0, z1
        divide = 1 - divide
    if elevation < divide:
        elevation /= divide
        return down, z0, elevation
    elevation = (elevation - divide) / (1 - divide)
    return up, z0, elevation


def streamline_tracking(fractures, elements, aperture, z0, f: int, elevation, ds, max_length, backward=False):
    """andfn/dfn.py:2643-2722.  Returns (segments, segment fractures, segment
    velocities, last element index or -1), each segment a complex array."""
    streamline, streamline_frac, velocity = [], [], []
    element = -1
    z0 = np.complex128(z0)
    z_start = z0
    while True:
        ds_frac = fractures[f]["radius"] * ds
        length = sum(len(s) for s in streamline)
        psi = [z_start]
        w = [calc_velocity(fractures, elements, aperture, f, z0)]
        z1 = runge_kutta(fractures, elements, z0, f, ds_frac, backward)
        if np.isnan(np.real(z1)) or np.isnan(np.imag(z1)):
            break
        z3, element = check_streamline_exit(fractures, elements, z0, z1, f)
        while z3 is None:
            psi.append(z1)
            w.append(calc_velocity(fractures, elements, aperture, f, z1))
            z0 = z1
            z1 = runge_kutta(fractures, elements, z0, f, ds_frac, backward)
            if np.isnan(np.real(z1)) or np.isnan(np.imag(z1)):
                z3 = z0
                break
            z3, element = check_streamline_exit(fractures, elements, z0, z1, f)
            if len(psi) > max_length - length:
                z3 = z1
                break
        psi.append(z3)
        w.append(calc_velocity(fractures, elements, aperture, f, z3))
        streamline.append(np.array(psi, np.complex128))
        streamline_frac.append(f)
        velocity.append(np.array(w, np.float64))
        if element >= 0 and int(elements[element]["_type"]) == 0:
            z3d = map_2d_to_3d(fractures, f, z3)
            f_old = f
            el = elements[element]
            f = int(el["frac1"]) if f == int(el["frac0"]) else int(el["frac0"])
            z0, z_start, elevation = get_exit_intersection(fractures, elements, z3d, element, f, f_old, elevation)
        else:
            break
    return streamline, streamline_frac, velocity, element


def travel_time_and_length(streamline, velocity):
    """andfn/dfn.py:2848-2903: sum over segments of |dz| / v (velocity at the
    start of each step) and of |dz|, NaN points removed."""
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
