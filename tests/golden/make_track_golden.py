"""Writes the golden vectors of streamline tracking by running the reference itself.

Run in a container where the reference source tree is available (its path is
the first argument, or $ANDFN_REFERENCE; further arguments name the cases
to write, all by default); the GPU machines never run this
script, they only read the ``track_*.npz`` files it writes next to itself.

For the converged state of two solve cases (the last k of ``mixed.npz``, which
holds every element type, and of ``c1_seed3.npz``) the network is rebuilt with
the reference's API, solved again with the same constants (the result is
checked to equal the stored records), unconsolidated into its objects
(DFN.unconsolidate_dfn(hpc=True)), given apertures, and traced with the
reference's own ``DFN.streamline_tracking`` (andfn/dfn.py:2643-2722) from
seeded start points (numpy complex scalars: the impermeable circle's calc_w,
impermeable_object.py:148-154, takes any other scalar for an array), forward
and backward.  Stored per trace: every point,
its segment index, the segment's fracture, the velocities, the last element
(-1 for the reference's False) and ``DFN.get_travel_time_and_length``.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

from make_golden import build_c1, build_mixed, consolidated, import_reference, reference_path  # noqa: E402

CASES = (("mixed", 21, 12, 0.02, 150), ("c1_seed3", 22, 16, 0.01, 300), ("c1_seed13", 23, 16, 0.01, 300))


def main():
    only = set(sys.argv[2:])  # case names to (re)write; all when none are given
    andfn = import_reference(reference_path(sys.argv[:2]))
    from andfn.hpc.hpc_solve import solve as hpc_solve
    for name, seed, npart, ds, max_length in CASES:
        if only and name not in only:
            continue
        g = np.load(os.path.join(HERE, f"{name}.npz"), allow_pickle=True)
        k = int(np.asarray(g["its"]).max())
        dfn = build_mixed(andfn) if name == "mixed" else build_c1(andfn, int(name.split("seed")[1]))
        F, E = consolidated(dfn)
        c = g[f"constants_{k}"][()]
        hpc_solve(F, E, int(g["D"]), c, dfn.ntype_element)
        Fo, Eo = g[f"F_out_{k}"], g[f"E_out_{k}"]
        mc = Eo["coef"].shape[1]
        assert np.array_equal(E["coef"][:, :mc], Eo["coef"]) and np.array_equal(F["constant"], Fo["constant"])
        dfn.fractures_struc_array_hpc, dfn.elements_struc_array_hpc = F, E
        dfn.unconsolidate_dfn(hpc=True)
        rng = np.random.default_rng(seed)
        aperture = 10 ** rng.uniform(-4, -3, len(F))
        for fr, a in zip(dfn.fractures, aperture):
            fr.aperture = a
        pf = rng.integers(0, len(F), npart)
        pz = np.sqrt(rng.uniform(0.0, 0.8, npart)) * F["radius"][pf] * np.exp(1j * rng.uniform(0, 2 * np.pi, npart))
        pe = rng.uniform(0.0, 1.0, npart)
        pb = (np.arange(npart) % 2).astype(bool)
        out = {"k": k, "aperture": aperture, "start_frac": pf, "start_z": pz, "start_elev": pe,
               "backward": pb, "ds": ds, "max_length": max_length}
        pts, seg, segf, vel, npts, nseg, elem, tt, tl = [], [], [], [], [], [], [], [], []
        for i in range(npart):
            s, sf, v, e = dfn.streamline_tracking(np.complex128(pz[i]), dfn.fractures[pf[i]], float(pe[i]), ds,
                                                  max_length, bool(pb[i]))
            fids = [int(f._id) for f in sf]
            for j, (ss, vv) in enumerate(zip(s, v)):
                pts.append(np.asarray(ss, np.complex128))
                vel.append(np.asarray(vv, np.float64))
                seg.append(np.full(len(ss), j, np.int64))
                segf.append(np.full(len(ss), fids[j], np.int64))
            npts.append(sum(len(ss) for ss in s))
            nseg.append(len(s))
            elem.append(-1 if e is False else int(e._id))
            if len(s):
                t, le = dfn.get_travel_time_and_length([list(ss) for ss in s], [list(vv) for vv in v])
            else:
                t, le = 0.0, 0.0
            tt.append(t)
            tl.append(le)
        out.update(points=np.concatenate(pts), point_seg=np.concatenate(seg), point_frac=np.concatenate(segf),
                   velocity=np.concatenate(vel), npoints=np.array(npts), nseg=np.array(nseg),
                   element=np.array(elem), travel_time=np.array(tt), travel_length=np.array(tl))
        path = os.path.join(HERE, f"track_{name}.npz")
        np.savez_compressed(path, **out)
        print(f"track_{name}: {npart} traces, points {npts}, segments {nseg}, elements {elem} "
              f"-> {path} ({os.path.getsize(path) // 1024} KB)")


if __name__ == "__main__":
    main()
