"""Golden fingerprints of the reference's own solve on the two large networks
the benchmark measures.

Run in a container where the reference source tree is available: its path
is the first argument, or $ANDFN_REFERENCE.  The GPU machines never run this
script; they only read the ``bench_*.npz`` files it writes next to itself.

Networks (rebuilt on every machine by andfn_b200.network from their seeds;
the fixture stores a SHA-256 of the input records so a test can tell that it
solves the same network):

* ``bench_c2``: the plain-solve network -- 5,500 power-law/Fisher discs in a
  50 m cube (seed 5), the largest cluster joining both head planes (2,118
  fractures, 5,376 elements), ncoef 20, nint 40;
* ``bench_c5``: the large network -- 20,000 discs (radii 1-40 m) in a 200 m
  cube (seed 11), largest spanning cluster (2,588 fractures) plus 100
  impermeable circles, ncoef 30, nint 60.

For each its in the case's list the reference's ``andfn.hpc.hpc_solve.solve``
runs with MAX_ITERATIONS = its (MAX_ERROR 1e-8, so the longest run stops at
convergence) on records of the reference's own dtypes.  The full outputs are
too large to keep, so each is stored as
  * a SHA-256 of every output field (the bit-exact check: the oracle must
    produce the same bytes),
  * the full q, fracture constants, errors, ncoef and nint,
  * the coefficients of 256 sampled elements (diagnostics when a hash
    differs, and a direct value check),
  * the iteration statistics the reference logs.
For bench_c2 the converged state also gets the reference's heads Re(Omega)/t
(hpc_fracture.calc_omega) at 10,000 seeded points.
"""
from __future__ import annotations

import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, ROOT)

from make_golden import import_reference, reference_path, repack  # noqa: E402

FIELDS = ("coef", "q", "error", "error_old", "error_old2", "error_coef", "dpsi_corr", "thetas", "ncoef", "nint")
NSAMPLE = 256


def digest(a: np.ndarray) -> str:
    """SHA-256 of an array's bytes in C order (little-endian as stored)."""
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def records_digest(F, E) -> str:
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(F).tobytes())
    h.update(np.ascontiguousarray(E).tobytes())
    return h.hexdigest()


def output_fingerprint(F, E, prefix, sample):
    out = {}
    for name in FIELDS:
        out[f"{prefix}sha_{name}"] = np.array(digest(E[name]))
    out[f"{prefix}sha_constant"] = np.array(digest(F["constant"]))
    for name in ("q", "error", "error_coef", "ncoef", "nint"):
        out[f"{prefix}{name}"] = np.array(E[name])
    out[f"{prefix}constant"] = np.array(F["constant"])
    out[f"{prefix}coef_sample"] = np.array(E["coef"][sample])
    out[f"{prefix}dpsi_corr_sample"] = np.array(E["dpsi_corr"][sample])
    return out


def case_networks():
    from andfn_b200 import network as nw
    return {
        "bench_c2": (lambda: nw.to_records(nw.power_law_fisher(5, nf=5500, L=50.0, ncoef=20, nint=40)), 20,
                     [1, 3, 200], 10000),
        "bench_c5": (lambda: nw.to_records(nw.large_network()), 30, [1, 2], 0),
    }


def heads_points(F, E, n, seed):
    """Seeded points inside the fractures (0.95 R), away from wells and
    impermeable circles (whose interiors are NaN)."""
    rng = np.random.default_rng(seed)
    fr = rng.integers(0, len(F), n)
    z = F["radius"][fr] * 0.95 * np.sqrt(rng.uniform(size=n)) * np.exp(2j * np.pi * rng.uniform(size=n))
    for i in range(n):
        for k in range(F["nelements"][fr[i]]):
            el = F["elements"][fr[i]][k]
            while E["_type"][el] in (2, 4) and abs(z[i] - E["center"][el]) < 1.5 * E["radius"][el]:
                z[i] = F["radius"][fr[i]] * 0.95 * np.sqrt(rng.uniform()) * np.exp(2j * np.pi * rng.uniform())
    return fr.astype(np.int64), z


def run(andfn, name, make, ncoef, its_list, nheads):
    from andfn.element import element_dtype_hpc
    from andfn.fracture import fracture_dtype_hpc
    from andfn.hpc import hpc_fracture
    from andfn.hpc.hpc_solve import solve as hpc_solve

    from andfn_b200.records import default_constants
    Fc, Ec = make()
    if Fc["nelements"].max() > fracture_dtype_hpc["elements"].shape[0]:
        raise SystemExit(f"{name}: a fracture holds more elements than the reference's MAX_ELEMENTS")
    Fr, Er = repack(Fc, fracture_dtype_hpc), repack(Ec, element_dtype_hpc)
    rng = np.random.default_rng(99)
    sample = np.sort(rng.choice(len(Ec), size=min(NSAMPLE, len(Ec)), replace=False))
    out = {"input_sha": np.array(records_digest(Fc, Ec)), "nf": np.array(len(Fc)), "ne": np.array(len(Ec)),
           "its": np.array(its_list), "D": np.array(50), "sample": sample}
    for k in its_list:
        c = default_constants(MAX_ITERATIONS=k, MAX_ERROR=1e-8, MAX_NCOEF=ncoef)
        F1, E1 = Fr.copy(), Er.copy()
        t0 = time.perf_counter()
        hpc_solve(F1, E1, 50, c, np.zeros(6, np.int64))
        dt = time.perf_counter() - t0
        Fo, Eo = repack(F1, Fc.dtype), repack(E1, Ec.dtype)
        out.update(output_fingerprint(Fo, Eo, f"k{k}_", sample))
        out[f"k{k}_constants"] = c
        out[f"k{k}_seconds"] = np.array(dt)
        print(f"{name}: k={k} solved in {dt:.1f} s, max |coef| {np.abs(Eo['coef']).max():.3e}", flush=True)
        if nheads and k == its_list[-1]:
            fr, z = heads_points(Fo, Eo, nheads, seed=23)
            h = np.array([hpc_fracture.calc_omega(F1[fr[i]], z[i], E1).real / F1["t"][fr[i]] for i in range(nheads)])
            out["heads_frac"], out["heads_z"], out["heads_ref"], out["heads_k"] = fr, z, h, np.array(k)
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **out)
    print(f"{name}: {len(Fc)} fractures, {len(Ec)} elements -> {path} ({os.path.getsize(path) // 1024} KB)")


def main():
    andfn = import_reference(reference_path(sys.argv[:2]))
    only = set(sys.argv[2:])
    for name, (make, ncoef, its, nheads) in case_networks().items():
        if not only or name in only:
            run(andfn, name, make, ncoef, its, nheads)


if __name__ == "__main__":
    main()
