"""Seeded discrete-fracture networks in the reference's record format.

The solve's input is built on the host by the reference's model-building API;
this module restates that pipeline with numpy so that networks of any size
can be generated where the reference is not installed (benchmarks, GPU
tests).  It follows:

* fracture frames: andfn/fracture.py:60-68 (x = n x (n + e_x), or n x (n + (1,1,1)));
* pairwise intersections in list order with frac0 the earlier fracture:
  DFN.get_fracture_intersections (andfn/dfn.py:1393-1458) and
  geometry_functions.fracture_intersection / line_circle_intersection /
  shorten_line (andfn/geometry_functions.py:302-402, 974-993);
* constant-head boundaries cut by large bounding planes:
  set_head_boundary (andfn/geometry_functions.py:878-926);
* removal of fractures not connected to a boundary: check_connectivity
  (andfn/dfn.py:1674-1695, geometry_functions.py:1262-1294);
* element order bounding, impermeable circle, impermeable line, constant
  head, well, intersection with ids = index: DFN.get_elements
  (andfn/dfn.py:995-1063), and the record fields of consolidate_dfn
  (andfn/dfn.py:658-820).

Padding fields are zero (the reference leaves them uninitialised).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .records import element_dtype, fracture_dtype


@dataclass
class Element:
    type: int
    frac0: int
    frac1: int = -1
    ep0: tuple = (0j, 0j)
    ep1: tuple = (0j, 0j)
    radius: float = 0.0
    center: complex = 0j
    head: float = 0.0
    ncoef: int = 0
    nint: int = 0
    q: float = 0.0


@dataclass
class Network:
    centers: np.ndarray
    normals: np.ndarray
    radii: np.ndarray
    t: np.ndarray
    xvec: np.ndarray = None
    yvec: np.ndarray = None
    elements: list = field(default_factory=list)      # list of Element
    frac_elems: list = field(default_factory=list)    # per fracture: element indices in order


def frames(normals: np.ndarray):
    """x/y unit vectors of each fracture plane (andfn/fracture.py:60-68)."""
    n = np.asarray(normals, float)
    x = np.cross(n, n + np.array([1.0, 0.0, 0.0]))
    zero = np.linalg.norm(x, axis=-1) == 0
    if np.any(zero):
        x[zero] = np.cross(n[zero], n[zero] + np.array([1.0, 1.0, 1.0]))
    x = x / np.linalg.norm(x, axis=-1, keepdims=True)
    y = np.cross(n / np.linalg.norm(n, axis=-1, keepdims=True), x)
    y = y / np.linalg.norm(y, axis=-1, keepdims=True)
    return x, y


def _dot(a, b):
    return a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1] + a[..., 2] * b[..., 2]


def _to2d(p, c, xv, yv):
    d = p - c
    return _dot(d, xv) + 1j * _dot(d, yv)


def _to3d(z, c, xv, yv):
    return np.real(z)[..., None] * xv + np.imag(z)[..., None] * yv + c


def _line_circle(z0, z1, R):
    """Vectorised line_circle_intersection (geometry_functions.py:359-402)."""
    dx = np.real(z1 - z0)
    dy = np.imag(z1 - z0)
    ok = np.ones(z0.shape, bool)
    a_out = np.zeros(z0.shape, complex)
    b_out = np.zeros(z0.shape, complex)
    vert = dx == 0
    with np.errstate(divide="ignore", invalid="ignore"):
        x = np.real(z0)
        y1 = np.sqrt(R ** 2 - x ** 2)
        a_v, b_v = x + 1j * y1, x - 1j * y1
        m = dy / np.where(vert, 1.0, dx)
        x0 = np.imag(z0) - m * np.real(z0)
        A = 1 + m ** 2
        B = 2 * x0 * m
        Cc = x0 ** 2 - R ** 2
        disc = B ** 2 - 4 * A * Cc
        sd = np.sqrt(np.where(disc < 0, 0.0, disc))
        x1 = (-B + sd) / (2 * A)
        x2 = (-B - sd) / (2 * A)
        a_n = x1 + 1j * (m * x1 + x0)
        b_n = x2 + 1j * (m * x2 + x0)
    a_out = np.where(vert, a_v, a_n)
    b_out = np.where(vert, b_v, b_n)
    ok = np.where(vert, True, disc >= 0)
    return ok, a_out, b_out


def plane_disc_intersections(c0, n0, x0v, y0v, R0, c1, n1, x1v, y1v, R1):
    """Vectorised fracture_intersection (geometry_functions.py:302-356).

    Returns (valid mask, endpoints in frame 0 [...,2], endpoints in frame 1)."""
    d = np.cross(n0, n1)
    dn2 = _dot(d, d)
    valid = dn2 >= 1e-14
    dn2s = np.where(valid, dn2, 1.0)
    cc0 = _dot(n0, c0)
    cc1 = _dot(n1, c1)
    p0 = (cc0[..., None] * np.cross(n1, d) + cc1[..., None] * np.cross(d, n0)) / dn2s[..., None]
    p1 = p0 + d
    z00, z01 = _to2d(p0, c0, x0v, y0v), _to2d(p1, c0, x0v, y0v)
    z10, z11 = _to2d(p0, c1, x1v, y1v), _to2d(p1, c1, x1v, y1v)
    ok0, a0, b0 = _line_circle(z00, z01, R0)
    ok1, a1, b1 = _line_circle(z10, z11, R1)
    valid &= ok0 & ok1
    cand = np.stack([_to3d(a0, c0, x0v, y0v), _to3d(b0, c0, x0v, y0v),
                     _to3d(a1, c1, x1v, y1v), _to3d(b1, c1, x1v, y1v)], axis=-2)  # [...,4,3]
    in0 = np.linalg.norm(cand - c0[..., None, :], axis=-1) <= (R0[..., None] + 1e-8)
    in1 = np.linalg.norm(cand - c1[..., None, :], axis=-1) <= (R1[..., None] + 1e-8)
    inside = in0 & in1
    valid &= inside.sum(-1) == 2
    # first two valid candidates in order
    idx = np.argsort(~inside, axis=-1, kind="stable")[..., :2]
    pa = np.take_along_axis(cand, idx[..., 0:1, None], axis=-2)[..., 0, :]
    pb = np.take_along_axis(cand, idx[..., 1:2, None], axis=-2)[..., 0, :]
    e0 = np.stack([_to2d(pa, c0, x0v, y0v), _to2d(pb, c0, x0v, y0v)], axis=-1)
    e1 = np.stack([_to2d(pa, c1, x1v, y1v), _to2d(pb, c1, x1v, y1v)], axis=-1)
    return valid, e0, e1


def shorten(ep, se):
    """shorten_line (geometry_functions.py:974-993)."""
    c = (ep[..., 0] + ep[..., 1]) / 2
    return np.stack([c + (ep[..., 0] - c) * se, c + (ep[..., 1] - c) * se], axis=-1)


def _candidate_pairs(centers, radii):
    """All i < k whose discs may touch (|c_i - c_k| <= r_i + r_k), in (i, k) order."""
    from scipy.spatial import cKDTree
    tree = cKDTree(centers)
    pairs = tree.query_pairs(2.0 * float(radii.max()), output_type="ndarray")
    if len(pairs) == 0:
        return pairs.reshape(0, 2)
    pairs = np.sort(pairs, axis=1)
    i, k = pairs[:, 0], pairs[:, 1]
    d = np.linalg.norm(centers[i] - centers[k], axis=1)
    pairs = pairs[d <= radii[i] + radii[k]]
    order = np.lexsort((pairs[:, 1], pairs[:, 0]))
    return pairs[order]


def gpu_disc_intersections(centers, normals, xv, yv, radii, se_factor, device=-1):
    """Disc-disc intersection segments of every pair i < k on the GPU
    (andfn_b200_disc_intersections): the pairs sorted by (i, k) and the
    shortened endpoints in both discs' frames, bit for bit what
    _candidate_pairs + plane_disc_intersections + shorten compute."""
    import ctypes

    from . import _ffi
    L = _ffi.lib()
    P = ctypes.c_void_p
    arrs = [np.ascontiguousarray(a, np.float64) for a in (centers, normals, xv, yv)]
    r = np.ascontiguousarray(radii, np.float64)
    nf = len(r)
    if any(a.shape != (nf, 3) for a in arrs):
        raise ValueError("centers, normals, xv and yv must be nf x 3")
    cap = max(16, 8 * nf)
    for _ in range(2):
        pairs = np.empty((cap, 2), np.int64)
        e0 = np.empty((cap, 2), np.complex128)
        e1 = np.empty((cap, 2), np.complex128)
        n = ctypes.c_int64()
        rc = L.andfn_b200_disc_intersections(int(device), nf, *[a.ctypes.data_as(P) for a in arrs],
                                             r.ctypes.data_as(P), float(se_factor), cap, pairs.ctypes.data_as(P),
                                             e0.ctypes.data_as(P), e1.ctypes.data_as(P), ctypes.byref(n))
        if rc == 0:
            return pairs[: n.value], e0[: n.value], e1[: n.value]
        if rc == 11 and n.value > cap:
            cap = n.value
            continue
        raise _ffi.AndfnError(rc, L.andfn_b200_geometry_last_error().decode())
    raise RuntimeError("disc_intersections: segment count changed between calls")


def gpu_clusters(nf, pairs, device=-1):
    """Connected components of the fracture graph given by pairs (i, k) on the
    GPU (andfn_b200_clusters): each fracture's label is the smallest fracture
    index of its component."""
    import ctypes

    from . import _ffi
    L = _ffi.lib()
    P = ctypes.c_void_p
    pr = np.ascontiguousarray(np.asarray(pairs, np.int64).reshape(-1, 2))
    out = np.empty(int(nf), np.int64)
    rc = L.andfn_b200_clusters(int(device), int(nf), len(pr), pr.ctypes.data_as(P), out.ctypes.data_as(P))
    if rc:
        raise _ffi.AndfnError(rc, L.andfn_b200_geometry_last_error().decode())
    return out


def build(centers, normals, radii, t, ncoef, nint, se_factor=0.9, heads=((0.0, 1.0),), axis=0, box=None,
          keep="connected", device=None):
    """Intersections, constant-head boundaries and connectivity for given discs.

    heads: ((coordinate, head), ...) of planes normal to ``axis`` cutting the
    box (the reference's set_constant_head_boundary with a plane of radius L).
    keep: "connected" (reference check_connectivity), "largest_spanning"
    (only the largest cluster that joins two different heads), or "all".
    device: None computes the disc-disc intersections on the host (numpy);
    a CUDA ordinal (-1: the current one) computes them, and the clusters, on
    the GPU, with the same results.
    """
    centers = np.asarray(centers, float)
    normals = np.asarray(normals, float)
    radii = np.asarray(radii, float)
    t = np.asarray(t, float)
    nf = len(radii)
    xv, yv = frames(normals)
    nrm = normals / np.linalg.norm(normals, axis=-1, keepdims=True)
    net = Network(centers, nrm, radii, t, xv, yv)
    # bounding circles (fracture.py:68-74)
    for f in range(nf):
        net.elements.append(Element(type=1, frac0=f, radius=float(radii[f]), ncoef=ncoef, nint=nint))
        net.frac_elems.append([f])
    # intersections
    if device is None:
        pairs = _candidate_pairs(centers, radii)
        if len(pairs):
            i, k = pairs[:, 0], pairs[:, 1]
            valid, e0, e1 = plane_disc_intersections(centers[i], normals[i], xv[i], yv[i], radii[i],
                                                     centers[k], normals[k], xv[k], yv[k], radii[k])
            e0 = shorten(e0, se_factor)
            e1 = shorten(e1, se_factor)
            sel = np.nonzero(valid)[0]
            pairs, e0, e1 = pairs[sel], e0[sel], e1[sel]
    else:
        pairs, e0, e1 = gpu_disc_intersections(centers, normals, xv, yv, radii, se_factor, device)
    for p in range(len(pairs)):
        a, b = int(pairs[p, 0]), int(pairs[p, 1])
        net.elements.append(Element(type=0, frac0=a, frac1=b, ep0=(e0[p, 0], e0[p, 1]),
                                    ep1=(e1[p, 0], e1[p, 1]), ncoef=ncoef, nint=nint))
        el = len(net.elements) - 1
        net.frac_elems[a].append(el)
        net.frac_elems[b].append(el)
    # constant-head planes (set_head_boundary): a disc of radius L normal to the axis
    if box is not None:
        L = float(box)
        for coord, head in heads:
            sc = np.full(3, L / 2)
            sc[axis] = coord
            sn = np.zeros(3)
            sn[axis] = 1.0
            sx, sy = frames(sn[None])
            R = L
            near = np.sum((centers - sc) ** 2, axis=1) <= (R + radii) ** 2
            idx = np.nonzero(near)[0]
            if len(idx) == 0:
                continue
            nS = len(idx)
            valid, _, e1 = plane_disc_intersections(
                np.repeat(sc[None], nS, 0), np.repeat(sn[None], nS, 0), np.repeat(sx, nS, 0),
                np.repeat(sy, nS, 0), np.full(nS, R), centers[idx], normals[idx], xv[idx], yv[idx], radii[idx])
            e1 = shorten(e1, se_factor)
            for p in np.nonzero(valid)[0]:
                f = int(idx[p])
                net.elements.append(Element(type=3, frac0=f, ep0=(e1[p, 0], e1[p, 1]), head=float(head),
                                            ncoef=ncoef, nint=nint))
                net.frac_elems[f].append(len(net.elements) - 1)
    if keep != "all":
        net = _prune(net, keep, device)
    return net


def _clusters(net, device=None):
    """Cluster label of every fracture: the smallest fracture index of its
    connected component (on the GPU with device set, andfn_b200_clusters)."""
    nf = len(net.radii)
    if device is not None:
        pairs = np.array([(e.frac0, e.frac1) for e in net.elements if e.type == 0], np.int64).reshape(-1, 2)
        return gpu_clusters(nf, pairs, device)
    par = np.arange(nf)

    def find(x):
        while par[x] != x:
            par[x] = par[par[x]]
            x = par[x]
        return x
    for e in net.elements:
        if e.type == 0:
            a, b = find(e.frac0), find(e.frac1)
            par[max(a, b)] = min(a, b)  # the smaller index stays the root
    return np.array([find(f) for f in range(nf)])


def _prune(net, keep, device=None):
    root = _clusters(net, device)
    bnd = {}
    for e in net.elements:
        if e.type in (2, 3) and not np.isnan(e.head):  # a NaN head: prescribed discharge, no head boundary
            bnd.setdefault(root[e.frac0], set()).add(e.head)
    if keep == "connected":
        keep_roots = set(bnd)
    elif keep == "largest_spanning":
        span = [r for r, h in bnd.items() if len(h) >= 2]
        if not span:
            keep_roots = set()
        else:
            sizes = {r: int(np.sum(root == r)) for r in span}
            keep_roots = {max(span, key=lambda r: (sizes[r], -r))}
    else:
        raise ValueError(keep)
    kept = [f for f in range(len(net.radii)) if root[f] in keep_roots]
    newid = {f: i for i, f in enumerate(kept)}
    out = Network(net.centers[kept], net.normals[kept], net.radii[kept], net.t[kept], net.xvec[kept],
                  net.yvec[kept])
    remap = {}
    for f in kept:
        lst = []
        for el in net.frac_elems[f]:
            e = net.elements[el]
            if e.type == 0 and not (e.frac0 in newid and e.frac1 in newid):
                continue
            if el not in remap:
                e2 = Element(**{**e.__dict__})
                e2.frac0 = newid[e.frac0]
                e2.frac1 = newid[e.frac1] if e.type == 0 else -1
                out.elements.append(e2)
                remap[el] = len(out.elements) - 1
            lst.append(remap[el])
        out.frac_elems.append(lst)
    return out


def add_well(net, frac, center, radius, head, q=None):
    """A well on a fracture: head-specified (andfn/well.py), or, with q given,
    with that prescribed discharge (head NaN; an extension of the reference,
    whose wells prescribe a head)."""
    if q is None:
        e = Element(type=2, frac0=frac, radius=radius, center=complex(center), head=head)
    else:
        e = Element(type=2, frac0=frac, radius=radius, center=complex(center), head=float("nan"), q=float(q))
    net.elements.append(e)
    net.frac_elems[frac].append(len(net.elements) - 1)


def add_impermeable_circle(net, frac, center, radius, ncoef, nint):
    net.elements.append(Element(type=4, frac0=frac, radius=radius, center=complex(center), ncoef=ncoef,
                                nint=nint))
    net.frac_elems[frac].append(len(net.elements) - 1)


def add_impermeable_line(net, frac, ep, ncoef, nint):
    net.elements.append(Element(type=5, frac0=frac, ep0=(complex(ep[0]), complex(ep[1])), ncoef=ncoef,
                                nint=nint))
    net.frac_elems[frac].append(len(net.elements) - 1)


def to_records(net, max_ncoef=None, max_elements=None):
    """Element and fracture records, element order and ids as DFN.get_elements."""
    seen = []
    mark = set()
    for lst in net.frac_elems:
        for el in lst:
            if el not in mark:
                mark.add(el)
                seen.append(el)
    order = []
    for ty in (1, 4, 5, 3, 2, 0):
        order += [el for el in seen if net.elements[el].type == ty]
    newid = {el: i for i, el in enumerate(order)}
    ne, nf = len(order), len(net.radii)
    mc = max_ncoef or max(1, max(net.elements[el].ncoef for el in order))
    me = max_elements or max(1, max(len(lst) for lst in net.frac_elems))
    E = np.zeros(ne, element_dtype(mc))
    F = np.zeros(nf, fracture_dtype(me))
    for i, el in enumerate(order):
        e = net.elements[el]
        r = E[i]
        r["_id"] = i
        r["_type"] = e.type
        r["frac0"] = e.frac0
        r["frac1"] = e.frac1
        r["endpoints0"] = e.ep0
        r["endpoints1"] = e.ep1
        r["radius"] = e.radius
        r["center"] = e.center
        r["head"] = e.head
        r["phi"] = e.head * net.t[e.frac0] if e.type in (2, 3) else 0.0  # Fracture.phi_from_head
        r["q"] = e.q
        r["ncoef"] = e.ncoef
        r["nint"] = e.nint
    F["_id"] = np.arange(nf)
    F["t"] = net.t
    F["radius"] = net.radii
    F["center"] = net.centers
    F["normal"] = net.normals
    F["x_vector"] = net.xvec
    F["y_vector"] = net.yvec
    for f, lst in enumerate(net.frac_elems):
        if len(lst) > me:
            raise ValueError(f"fracture {f} has {len(lst)} elements > MAX_ELEMENTS {me}")
        F["elements"][f, : len(lst)] = [newid[el] for el in lst]
        F["nelements"][f] = len(lst)
    return F, E


# ---------------------------------------------------------------------------
# Seeded recipes
# ---------------------------------------------------------------------------
def uniform_discs(seed, nf=30, L=20.0, rmin=1.0, rmax=5.0, logt=(-5.0, 0.5), ncoef=10, nint=20,
                  se_factor=0.9, keep="connected", **kw):
    """nf discs in an L cube: per fracture, in this draw order, a centre
    U[0, L]^3, a normal N(0, I) normalised, a radius U[rmin, rmax] and
    log10 T ~ N(logt); constant heads 1 at x = 0 and 0 at x = L."""
    rng = np.random.default_rng(seed)
    c = np.empty((nf, 3))
    n = np.empty((nf, 3))
    r = np.empty(nf)
    t = np.empty(nf)
    for i in range(nf):
        c[i] = rng.uniform(0, L, 3)
        v = rng.normal(size=3)
        n[i] = v / np.linalg.norm(v)
        r[i] = rng.uniform(rmin, rmax)
        t[i] = 10 ** rng.normal(logt[0], logt[1])
    return build(c, n, r, t, ncoef, nint, se_factor, heads=((0.0, 1.0), (L, 0.0)), box=L, keep=keep, **kw)


def power_law_fisher(seed, nf, L, rmin=0.5, rmax=20.0, alpha=2.6, kappa=5.0, logt=(-5.0, 1.0), ncoef=20,
                     nint=40, se_factor=0.9, keep="largest_spanning", **kw):
    """nf discs in an L cube with power-law radii (pdf ~ r^-alpha on
    [rmin, rmax], inverse CDF), Fisher(kappa) normals about a random pole,
    log10 T ~ N(logt); heads 1 at x = 0 and 0 at x = L."""
    rng = np.random.default_rng(seed)
    a = alpha - 1.0
    u = rng.uniform(size=nf)
    r = rmin * (1 - u * (1 - (rmin / rmax) ** a)) ** (-1 / a)
    pole = rng.normal(size=3)
    pole /= np.linalg.norm(pole)
    w = 1 + np.log(np.exp(-2 * kappa) + (1 - np.exp(-2 * kappa)) * rng.uniform(size=nf)) / kappa
    phi = rng.uniform(0, 2 * np.pi, nf)
    tmp = np.array([1.0, 0, 0]) if abs(pole[0]) < 0.9 else np.array([0, 1.0, 0])
    e1 = np.cross(pole, tmp)
    e1 /= np.linalg.norm(e1)
    e2 = np.cross(pole, e1)
    s = np.sqrt(np.clip(1 - w ** 2, 0, None))
    n = w[:, None] * pole + s[:, None] * (np.cos(phi)[:, None] * e1 + np.sin(phi)[:, None] * e2)
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    c = rng.uniform(0, L, (nf, 3))
    t = 10 ** rng.normal(logt[0], logt[1], nf)
    order = np.argsort(-r, kind="stable")  # large fractures first
    return build(c[order], n[order], r[order], t[order], ncoef, nint, se_factor,
                 heads=((0.0, 1.0), (L, 0.0)), box=L, keep=keep, **kw)


def to_records_batch(nets):
    """Records of several networks with one shared layout (the batch API needs
    a common MAX_NCOEF / MAX_ELEMENTS)."""
    mc = max(max(1, max(e.ncoef for e in n.elements)) for n in nets)
    me = max(max(1, max(len(lst) for lst in n.frac_elems)) for n in nets)
    return [to_records(n, max_ncoef=mc, max_elements=me) for n in nets]


def _seg_dist(z, a, b):
    d = b - a
    t = 0.0 if d == 0 else min(1.0, max(0.0, ((z - a) * d.conjugate()).real / abs(d) ** 2))
    return abs(z - (a + t * d))


def place_wells(net, rng, n, radius=0.05, head=(0.0, 1.0), clearance=10.0, rim=0.8, tries=200, q=None):
    """n wells at uniform random points (inside rim * R) of random fractures,
    at least clearance * radius away from every line element of that fracture
    and from the other wells; head-specified with head U[head], or, when q is
    a range, with a prescribed discharge U[q]."""
    nf = len(net.radii)
    for _ in range(n):
        for _t in range(tries):
            f = int(rng.integers(0, nf))
            R = float(net.radii[f])
            z = rim * R * np.sqrt(rng.uniform()) * np.exp(2j * np.pi * rng.uniform())
            ok = True
            for el in net.frac_elems[f]:
                e = net.elements[el]
                if e.type in (0, 3, 5):
                    ep = e.ep1 if (e.type == 0 and e.frac1 == f) else e.ep0
                    ok = _seg_dist(z, complex(ep[0]), complex(ep[1])) > clearance * radius
                elif e.type in (2, 4):
                    ok = abs(z - e.center) > clearance * radius + e.radius
                if not ok:
                    break
            if ok:
                if q is None:
                    add_well(net, f, z, radius, float(rng.uniform(*head)))
                else:
                    add_well(net, f, z, radius, float("nan"), q=float(rng.uniform(*q)))
                break


def batch_realization(seed, L=40.0, nf_range=(200, 800), wells=4, ncoef=15, nint=30, well_q=(-1e-4, 1e-4), **kw):
    """One realization of the batched workload: N_gen ~ U{200..800} discs drawn
    as power_law_fisher in an L cube, head planes 1 / 0 at x = 0 / L, then
    `wells` wells (radius 0.05 m) with a prescribed discharge U[well_q]
    (m^3/s) at random points of random fractures of the clusters that touch
    a head plane (the fractures kept, as check_connectivity does: a well in a
    cluster without a head boundary would have no steady state).  With
    well_q=None the wells are head-specified (head U[0, 1]) and placed before
    the pruning, so clusters joined to a well are kept too."""
    rng = np.random.default_rng([seed, 7])
    nf = int(rng.integers(nf_range[0], nf_range[1] + 1))
    net = power_law_fisher(seed, nf, L, ncoef=ncoef, nint=nint, keep="all", **kw)
    if well_q is None:
        place_wells(net, rng, wells)
        return _prune(net, "connected")
    net = _prune(net, "connected")
    if len(net.radii):
        place_wells(net, rng, wells, q=well_q)
    return net


def place_impermeable_circles(net, rng, n, rmin=1.0, rmax=3.0, ncoef=30, nint=60, clearance=1.2, tries=500):
    """n impermeable circles (radius U[rmin, rmax]) at random points of random
    fractures, inside the fracture and clear of its line elements and of the
    other circles."""
    nf = len(net.radii)
    placed = 0
    for _ in range(tries * n):
        if placed == n:
            break
        f = int(rng.integers(0, nf))
        R = float(net.radii[f])
        r = float(rng.uniform(rmin, rmax))
        if R < 2.5 * r:
            continue
        z = (R - 1.5 * r) * np.sqrt(rng.uniform()) * np.exp(2j * np.pi * rng.uniform())
        ok = True
        for el in net.frac_elems[f]:
            e = net.elements[el]
            if e.type in (0, 3, 5):
                ep = e.ep1 if (e.type == 0 and e.frac1 == f) else e.ep0
                ok = _seg_dist(z, complex(ep[0]), complex(ep[1])) > clearance * r
            elif e.type in (2, 4):
                ok = abs(z - e.center) > clearance * (r + e.radius)
            if not ok:
                break
        if ok:
            add_impermeable_circle(net, f, z, r, ncoef, nint)
            placed += 1
    return placed


def large_network(seed=11, nf=20000, L=200.0, n_imp=100, ncoef=30, nint=60):
    """The large single-network workload: nf power-law/Fisher discs (radii
    1-40 m) in an L cube, the largest cluster joining both head planes, plus
    n_imp impermeable circles (radius 1-3 m) on random fractures of it."""
    net = power_law_fisher(seed, nf, L, rmin=1.0, rmax=40.0, ncoef=ncoef, nint=nint)
    rng = np.random.default_rng([seed, 13])
    place_impermeable_circles(net, rng, n_imp, ncoef=ncoef, nint=nint)
    return net
