"""Writes the golden vectors of the solve by running the reference itself.

Run in a container where the reference source tree is available: its path
is the first argument, or the environment variable ANDFN_REFERENCE when no
argument is given.  The GPU machines never run this script; they only read
the .npz files it writes next to itself.

For every case the reference builds a seeded network through its public API
(Fracture, DFN.get_fracture_intersections, set_constant_head_boundary,
check_connectivity, ConstantHeadLine, Well, ImpermeableCircle/Line),
consolidates it (DFN.consolidate_dfn(hpc=True)) and then calls its own
``andfn.hpc.hpc_solve.solve`` with MAX_ITERATIONS = k for several k.

The reference's consolidation leaves several record fields uninitialised
(np.empty at andfn/dfn.py:675,712-715): they are zero-filled before solving
(coef beyond ncoef, old_coef, dpsi_corr, thetas, error_old, error_old2,
error_coef), which is the documented precondition of every case here.

Each case file holds the input records, the output records after each k, the
solver constants, and for converged cases heads Re(Omega)/t at random points
computed with the reference's hpc_fracture.calc_omega.
"""
from __future__ import annotations

import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def reference_path(argv):
    """The reference source tree: argv[1], else $ANDFN_REFERENCE."""
    path = argv[1] if len(argv) > 1 else os.environ.get("ANDFN_REFERENCE")
    if not path or not os.path.isdir(os.path.join(path, "andfn")):
        sys.exit(f"usage: {os.path.basename(argv[0])} REFERENCE_TREE (or set ANDFN_REFERENCE); "
                 f"the tree must contain the andfn package (got {path!r})")
    return path


def import_reference(path):
    for name in ("pyvista", "h5py", "matplotlib", "matplotlib.colors", "matplotlib.tri", "matplotlib.pyplot"):
        sys.modules.setdefault(name, types.ModuleType(name))
    sys.modules["matplotlib.colors"].LinearSegmentedColormap = type(
        "LinearSegmentedColormap", (), {"from_list": staticmethod(lambda *a, **k: None)})
    sys.modules["matplotlib.tri"].Triangulation = object
    sys.path.insert(0, path)
    os.environ.setdefault("NUMBA_CACHE_DIR", os.path.join(HERE, ".numba_cache"))
    import logging

    import andfn  # noqa: F401
    logging.getLogger("andfn").setLevel("WARNING")
    return andfn


def compact_dtypes(E, F):
    """Smallest record dtypes (same field order) that hold this network."""
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from andfn_b200.records import element_dtype, fracture_dtype
    mc = int(max(E["ncoef"].max(), 1))
    me = int(max(F["nelements"].max(), 1))
    return element_dtype(mc), fracture_dtype(me)


def repack(a, dtype):
    out = np.zeros(len(a), dtype)
    for name in dtype.names:
        src = a[name]
        dst = out[name]
        if src.ndim == 1:
            dst[:] = src
        else:
            n = min(src.shape[1], dst.shape[1])
            dst[:, :n] = src[:, :n]
    return out


def build_c1(andfn, seed, nf=30, L=20.0, ncoef=10, nint=20, **kw):
    """30 discs in a 20 m cube, constant heads 1 / 0 on x = 0 / x = L."""
    rng = np.random.default_rng(seed)
    fr = []
    for i in range(nf):
        c = rng.uniform(0, L, 3)
        n = rng.normal(size=3)
        n /= np.linalg.norm(n)
        r = rng.uniform(1, 5)
        t = 10 ** rng.normal(-5, 0.5)
        fr.append(andfn.Fracture(f"{i}", t, r, c, n, ncoef=ncoef, nint=nint))
    dfn = andfn.DFN("c1", **kw)
    dfn.add_fracture(fr)
    dfn.get_fracture_intersections(ncoef, nint)
    dfn.set_constant_head_boundary(np.array([0, L / 2, L / 2]), np.array([1.0, 0, 0]), L, 1.0, ncoef=ncoef, nint=nint)
    dfn.set_constant_head_boundary(np.array([L, L / 2, L / 2]), np.array([1.0, 0, 0]), L, 0.0, ncoef=ncoef, nint=nint)
    dfn.get_elements()
    dfn.check_connectivity()
    return dfn


def build_mixed(andfn, ncoef=10, nint=20, **kw):
    """Four fractures with every element type: intersections, bounding
    circles, two constant-head lines, a well, an impermeable circle and an
    impermeable line (geometry after the reference's examples/template.py)."""
    Fr = andfn.fracture.Fracture
    f0 = Fr("a", 1, radius=0.7, center=np.array([-0.7, 0.1, -0.3]), normal=np.array([-0.2, 0.4, -0.9]),
            ncoef=ncoef, nint=nint)
    f1 = Fr("b", 2, radius=1.0, center=np.array([-0.6, -0.61, -0.7]), normal=np.array([-0.6, -0.5, 0.6]),
            ncoef=ncoef, nint=nint)
    f2 = Fr("c", 3, radius=0.5, center=np.array([0.0, 0.0, -0.1]), normal=np.array([0.3, -0.8, -0.4]),
            ncoef=ncoef, nint=nint)
    f3 = Fr("d", 5, radius=0.7, center=np.array([-0.1, -1.0, 0.3]), normal=np.array([0.5, 0.0, 0.0]),
            ncoef=ncoef, nint=nint)
    andfn.const_head.ConstantHeadLine("ch0", np.array([0.3 + 0.2j, 0.2 - 0.3j]), 10.0, f3, ncoef, nint)
    andfn.const_head.ConstantHeadLine("ch1", np.array([-0.4 - 0.1j, -0.3 - 0.3j]), 2.0, f0, ncoef, nint)
    andfn.well.Well("w0", 0.05, -0.005 + 0.002j, 5.0, f3)
    andfn.impermeable_object.ImpermeableCircle("ic0", 0.12, 0.35 + 0.3j, f1, ncoef, nint)
    andfn.impermeable_object.ImpermeableLine("il0", np.array([-0.25 + 0.2j, -0.05 + 0.3j]), f2, ncoef, nint)
    dfn = andfn.DFN("mixed", **kw)
    dfn.add_fracture([f0, f1, f2, f3])
    dfn.get_fracture_intersections(ncoef, nint)
    dfn.get_elements()
    return dfn


def consolidated(dfn):
    dfn.get_elements()
    dfn.consolidate_dfn(hpc=True)
    E = dfn.elements_struc_array_hpc
    for i in range(len(E)):
        nc = E["ncoef"][i]
        E["coef"][i, nc:] = 0
    for name in ("old_coef", "dpsi_corr", "thetas", "error_old", "error_old2", "error_coef"):
        E[name] = 0
    return dfn.fractures_struc_array_hpc.copy(), E.copy()


def spanning(E, F):
    """True when one connected cluster (union-find over intersections)
    carries constant-head lines of two different heads, i.e. flow is not
    identically zero."""
    par = list(range(len(F)))

    def find(x):
        while par[x] != x:
            par[x] = par[par[x]]
            x = par[x]
        return x
    for i in np.nonzero(E["_type"] == 0)[0]:
        par[find(E["frac0"][i])] = find(E["frac1"][i])
    heads = {}
    for i in np.nonzero(E["_type"] == 3)[0]:
        heads.setdefault(find(E["frac0"][i]), set()).add(float(E["head"][i]))
    return any(len(v) >= 2 for v in heads.values())


def heads_points(andfn, F, E, npts, seed):
    from andfn.hpc import hpc_fracture
    rng = np.random.default_rng(seed)
    fr = rng.integers(0, len(F), npts)
    zs = np.empty(npts, np.complex128)
    for i in range(npts):
        R = F["radius"][fr[i]]
        while True:
            z = R * 0.95 * np.sqrt(rng.uniform()) * np.exp(2j * np.pi * rng.uniform())
            bad = False
            for k in range(F["nelements"][fr[i]]):
                el = F["elements"][fr[i]][k]
                if E["_type"][el] in (2, 4) and abs(z - E["center"][el]) < 1.5 * E["radius"][el]:
                    bad = True
            if not bad:
                break
        zs[i] = z
    h = np.array([hpc_fracture.calc_omega(F[fr[i]], zs[i], E).real / F["t"][fr[i]] for i in range(npts)])
    return fr.astype(np.int64), zs, h


def run_case(andfn, name, dfn, its, max_error=1e-8, max_ncoef=None, D=50, nheads=0):
    from andfn.hpc.hpc_solve import solve as hpc_solve
    F, E = consolidated(dfn)
    edt, fdt = compact_dtypes(E, F)
    if max_ncoef is not None and max_ncoef > E["ncoef"].max():
        from andfn_b200.records import element_dtype
        edt = element_dtype(int(max_ncoef))
    out = {"E_in": repack(E, edt), "F_in": repack(F, fdt), "its": np.array(its), "D": np.array(D)}
    cst = dfn.constants.copy()
    for k in its:
        c = cst.copy()
        c["MAX_ITERATIONS"] = k
        c["MAX_ERROR"] = max_error
        if max_ncoef is not None:
            c["MAX_NCOEF"] = max_ncoef
        F1, E1 = F.copy(), E.copy()
        hpc_solve(F1, E1, D, c, dfn.ntype_element)
        out[f"E_out_{k}"] = repack(E1, edt)
        out[f"F_out_{k}"] = repack(F1, fdt)
        out[f"constants_{k}"] = c
        if nheads and k == its[-1]:
            fr, zs, h = heads_points(andfn, F1, E1, nheads, seed=17)
            out["heads_frac"], out["heads_z"], out["heads_ref"] = fr, zs, h
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **out)
    print(f"{name}: {len(F)} fractures, {len(E)} elements, types {np.bincount(E['_type'], minlength=6)}, "
          f"its {its} -> {path} ({os.path.getsize(path) // 1024} KB)")


def main():
    andfn = import_reference(reference_path(sys.argv))
    # Seeds of the 30-disc recipe: flowing networks (one cluster joins both
    # heads) and one whose clusters touch a single head each (q = 0).
    seeds, trivial = [], []
    for seed in range(60):
        dfn = build_c1(andfn, seed, MAX_ERROR=1e-8, MAX_NCOEF=10)
        if dfn.number_of_fractures >= 2:
            F, E = consolidated(dfn)
            (seeds if spanning(E, F) else trivial).append(seed)
        if len(seeds) >= 3 and trivial:
            break
    print("spanning seeds", seeds, "trivial", trivial[:1])
    s0 = seeds[0]
    run_case(andfn, f"c1_seed{s0}", build_c1(andfn, s0, MAX_NCOEF=10), [1, 2, 5, 200], nheads=2000)
    for s in seeds[1:3]:
        run_case(andfn, f"c1_seed{s}", build_c1(andfn, s, MAX_NCOEF=10), [3, 200])
    run_case(andfn, f"c1_trivial_seed{trivial[0]}", build_c1(andfn, trivial[0], MAX_NCOEF=10), [2, 200])
    run_case(andfn, "mixed", build_mixed(andfn, MAX_NCOEF=10), [1, 3, 40], nheads=500)
    run_case(andfn, f"c1_seed{s0}_adaptive", build_c1(andfn, s0, MAX_NCOEF=10), [4, 8, 12], max_ncoef=40)


if __name__ == "__main__":
    main()
