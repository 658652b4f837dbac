"""Writes the golden vectors of the flow-field evaluations by running the reference itself.

Run in a container where the reference source tree is available (its path is
the first argument, or $ANDFN_REFERENCE); the GPU machines never run this
script, they only read the ``flow_*.npz`` files it writes next to itself.

For a converged state of the solve cases (the last k of ``mixed.npz``, which
holds every element type, and of ``c1_seed3.npz``) the reference's own
functions are called:

* ``andfn.hpc.hpc_fracture.sunflower_spiral(n_in, n_bnd)``;
* ``andfn.hpc.hpc_fracture.get_flow_nets(F, n_in, n_bnd, E)``, stored as its
  first column (the reference fills every column of row i with Omega(z_i))
  together with a check that all columns are equal, and its 3-D points;
* ``andfn.hpc.hpc_fracture.get_heads(F, E, z)`` on the same unit-disc points;
* ``andfn.hpc.hpc_fracture.calc_w(F[f], z, E)`` at random points inside
  random fractures (the complex discharge vector).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

from make_golden import import_reference, reference_path  # noqa: E402

N_IN, N_BND, N_W = 40, 12, 400


def case_state(name):
    g = np.load(os.path.join(HERE, f"{name}.npz"), allow_pickle=True)
    k = int(np.asarray(g["its"]).max())
    return g[f"F_out_{k}"].copy(), g[f"E_out_{k}"].copy(), k


def main():
    import_reference(reference_path(sys.argv[:2]))
    from andfn.hpc import hpc_fracture as hf
    for name, seed in (("mixed", 11), ("c1_seed3", 12)):
        F, E, k = case_state(name)
        out = {"k": k}
        zs = hf.sunflower_spiral(N_IN, N_BND)
        out["spiral"] = zs
        nets, p3 = hf.get_flow_nets(F, N_IN, N_BND, E)
        assert np.array_equal(nets, np.broadcast_to(nets[:, :, :1], nets.shape), equal_nan=True)
        out["flow_omega"], out["flow_pnts"] = nets[:, :, 0].copy(), p3
        heads, hp = hf.get_heads(F, E, zs)
        out["grid_heads"], out["grid_pnts"] = heads, hp
        rng = np.random.default_rng(seed)
        fr = rng.integers(0, len(F), N_W)
        r = np.sqrt(rng.uniform(0.0, 0.9, N_W)) * F["radius"][fr]
        th = rng.uniform(0.0, 2 * np.pi, N_W)
        z = r * np.exp(1j * th)
        w = np.array([hf.calc_w(F[f], zz, E) for f, zz in zip(fr, z)], np.complex128)
        out["w_frac"], out["w_z"], out["w_ref"] = fr, z, w
        path = os.path.join(HERE, f"flow_{name}.npz")
        np.savez_compressed(path, **out)
        print(path, {kk: np.shape(v) for kk, v in out.items()})


if __name__ == "__main__":
    main()
