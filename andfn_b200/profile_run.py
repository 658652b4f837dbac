"""Single runs of the benchmark workloads, for profiler captures.

``python -m andfn_b200.profile_run [MAX_ITERATIONS] [--adjoint | --batch]``

* default: one plain solve of the seeded 2,118-fracture network of bench.py
  through the one-call C ABI;
* ``--adjoint``: one forward solve plus the gradient of the bench objective
  (50 observation heads + outflow) with respect to log t (torch autograd);
* ``--batch``: one batched solve of the 256 bench realizations.
"""
import argparse
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def main():
    import numpy as np

    import bench

    import andfn_b200
    ap = argparse.ArgumentParser()
    ap.add_argument("iterations", nargs="?", type=int, default=None)
    g = ap.add_mutually_exclusive_group()
    g.add_argument("--adjoint", action="store_true")
    g.add_argument("--batch", action="store_true")
    a = ap.parse_args()
    if a.batch:
        recs = bench.build_batch()
        c = bench.batch_constants()
        if a.iterations:
            c["MAX_ITERATIONS"] = a.iterations
        st = andfn_b200.solve_batch(recs, 50, c)
        its = [s["iterations"] for s in st]
        print(f"realizations {len(st)} iterations max {max(its)} mean {np.mean(its):.1f}")
        return
    F, E = bench.build_network()
    c = bench.constants()
    if a.iterations:
        c["MAX_ITERATIONS"] = a.iterations
    if a.adjoint:
        import torch
        from andfn_b200.adjoint import DFNModel
        rng = np.random.default_rng(7)
        fr = rng.integers(0, len(F), 50)
        z = F["radius"][fr] * 0.9 * np.sqrt(rng.uniform(size=50)) * np.exp(2j * np.pi * rng.uniform(size=50))
        dev = "cuda:0"
        frt = torch.tensor(fr, device=dev)
        zt = torch.tensor(z, dtype=torch.complex128, device=dev)
        outlet = torch.tensor(np.nonzero((E["_type"] == 3) & (E["head"] == 0.0))[0], device=dev)
        m = DFNModel(F.copy(), E.copy(), c, 50, adjoint_tol=1e-8)
        lt = torch.tensor(np.log(F["t"]), device=dev, requires_grad=True)
        coef, q, C = m.solve(lt)
        h = m.heads(coef, q, C, lt, frt, zt)
        J = ((h - 0.5) ** 2).sum() + q[outlet].sum()
        J.backward()
        print(f"forward iterations {m.stats['iterations']} adjoint sweeps {m.adjoint_stats['iterations']} "
              f"residual {m.adjoint_stats['residual']:.2e}")
        m.close()
        return
    andfn_b200.solve(F, E, 50, c)
    st = andfn_b200.last_stats
    print(f"iterations {st['iterations']} status {st['status']} factor {st['ms_factor']:.1f} ms "
          f"iterate {st['ms_iterate']:.1f} ms")


if __name__ == "__main__":
    main()
