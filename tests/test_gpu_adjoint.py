"""Adjoint gradients d J / d log t against central finite differences.

J is the objective of the gradient workload: the squared misfit of heads at
observation points (observed = forward heads + N(0, 0.01)) plus the
discharge through the head-0 face (sum of q of the constant-head lines with
head 0).  Finite differences run the solve itself at t * exp(+-h) per
fracture: the GPU forward (every fracture) and the oracle (the reference's
algorithm on the CPU, a sample of fractures).  The solves run a fixed,
large number of iterations (MAX_ERROR below round-off), so J of the
iterate is a smooth function of log t and its difference quotient converges
to the fixed point's derivative.

Tolerance: |g_adjoint - g_fd| <= 1e-5 * max |g_fd| + 1e-12 * scale, the
north-star bound (1e-5 relative) taken against the largest gradient entry,
because entries of fractures that barely touch the flow are pure round-off
in the difference quotient.
"""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

H_FD = 1e-4


def _constants(ncoef, its=1500):
    from andfn_b200.records import default_constants
    return default_constants(MAX_ITERATIONS=its, MAX_ERROR=1e-300, MAX_NCOEF=ncoef)


def _points(F, n, seed):
    rng = np.random.default_rng(seed)
    fr = rng.integers(0, len(F), n)
    z = F["radius"][fr] * 0.9 * np.sqrt(rng.uniform(size=n)) * np.exp(2j * np.pi * rng.uniform(size=n))
    return fr, z


class Problem:
    def __init__(self, case, q_weight=1.0, seed=0):
        import torch
        from andfn_b200.adjoint import DFNModel
        g = load_golden(case)
        self.F, self.E = g["F_in"].copy(), g["E_in"].copy()
        self.c = _constants(int(self.E["ncoef"].max()))
        self.model = DFNModel(self.F.copy(), self.E.copy(), self.c, 50)
        self.logt0 = np.log(self.F["t"].astype(np.float64))
        fr, z = _points(self.F, 50, seed)
        self.fr_np, self.z_np = fr, z
        self.fr = torch.tensor(fr, dtype=torch.int64, device="cuda")
        self.z = torch.tensor(z, dtype=torch.complex128, device="cuda")
        self.outlet = np.nonzero((self.E["_type"] == 3) & (self.E["head"] == 0.0))[0]
        self.q_weight = q_weight
        h0 = self.heads_np(self.logt0)
        rng = np.random.default_rng(seed + 1)
        self.hobs = h0 + rng.normal(0.0, 0.01, len(h0))

    def heads_np(self, logt):
        import torch
        lt = torch.tensor(logt, dtype=torch.float64, device="cuda")
        coef, q, C = self.model.solve(lt)
        return self.model.heads(coef, q, C, lt, self.fr, self.z).cpu().numpy()

    def J_gpu(self, logt):
        import torch
        lt = torch.tensor(logt, dtype=torch.float64, device="cuda")
        coef, q, C = self.model.solve(lt)
        h = self.model.heads(coef, q, C, lt, self.fr, self.z)
        hobs = torch.tensor(self.hobs, device="cuda")
        return float(((h - hobs) ** 2).sum() + self.q_weight * q[self.outlet].sum())

    def grad_adjoint(self):
        import torch
        lt = torch.tensor(self.logt0, dtype=torch.float64, device="cuda", requires_grad=True)
        coef, q, C = self.model.solve(lt)
        h = self.model.heads(coef, q, C, lt, self.fr, self.z)
        hobs = torch.tensor(self.hobs, device="cuda")
        J = ((h - hobs) ** 2).sum() + self.q_weight * q[torch.tensor(self.outlet, device="cuda")].sum()
        J.backward()
        return lt.grad.cpu().numpy()

    def J_oracle(self, logt):
        from oracle import oracle as orc
        F, E = self.F.copy(), self.E.copy()
        t = np.exp(logt)
        F["t"] = t
        m = np.isin(E["_type"], (2, 3))
        E["phi"][m] = E["head"][m] * t[E["frac0"][m]]
        orc.solve(F, E, 50, self.c)
        h = orc.eval_heads(F, E, self.fr_np, self.z_np)
        return float(((h - self.hobs) ** 2).sum() + self.q_weight * E["q"][self.outlet].sum())


def _fd(J, logt0, fracs):
    g = np.zeros(len(fracs))
    for i, f in enumerate(fracs):
        lp, lm = logt0.copy(), logt0.copy()
        lp[f] += H_FD
        lm[f] -= H_FD
        g[i] = (J(lp) - J(lm)) / (2 * H_FD)
    return g


def _check(ga, gf, tag):
    err = np.abs(ga - gf)
    bound = 1e-5 * np.abs(gf).max() + 1e-30
    assert np.all(err <= bound), (tag, float(err.max() / np.abs(gf).max()), ga, gf)


@pytest.mark.parametrize("case", ["c1_seed3", "mixed"])
def test_adjoint_matches_gpu_finite_differences(case):
    P = Problem(case)
    ga = P.grad_adjoint()
    st = P.model.adjoint_stats
    assert st["status"] == 0, st
    fracs = np.arange(len(P.F))
    gf = _fd(P.J_gpu, P.logt0, fracs)
    _check(ga, gf, (case, "gpu"))


def test_adjoint_discharge_objective_matches_gpu_finite_differences():
    """J = discharge through the head-0 face only (the q path of the adjoint)."""
    P = Problem("c1_seed3", q_weight=1.0)

    import torch

    def J(logt):
        lt = torch.tensor(logt, dtype=torch.float64, device="cuda")
        coef, q, C = P.model.solve(lt)
        return float(q[P.outlet].sum())

    lt = torch.tensor(P.logt0, dtype=torch.float64, device="cuda", requires_grad=True)
    coef, q, C = P.model.solve(lt)
    q[torch.tensor(P.outlet, device="cuda")].sum().backward()
    ga = lt.grad.cpu().numpy()
    gf = _fd(J, P.logt0, np.arange(len(P.F)))
    _check(ga, gf, "discharge")


def test_adjoint_matches_oracle_finite_differences():
    """The same gradient against finite differences of the oracle solve (a
    sample of fractures, the largest gradients first)."""
    P = Problem("c1_seed3")
    ga = P.grad_adjoint()
    fracs = np.argsort(-np.abs(ga))[:6]
    gf = _fd(P.J_oracle, P.logt0, fracs)
    err = np.abs(ga[fracs] - gf)
    assert np.all(err <= 1e-5 * np.abs(ga).max()), (err / np.abs(ga).max(), ga[fracs], gf)


@pytest.mark.parametrize("inverse", [1, 0])
def test_adjoint_with_dense_tail_matches_gpu_finite_differences(inverse, monkeypatch):
    """A 588-fracture generated network (converges in 146 iterations) whose LU
    has a 364-row dense tail.  Discharge solves, forward and transposed,
    through the explicit inverse of the system and its transpose (1) or the
    triangular solves with the dense tail as a CTA cluster (0): gradient vs
    central differences of the GPU forward solve on the five largest entries
    (step 1e-4, fixed-iteration forward solves)."""
    monkeypatch.setenv("ANDFN_B200_EXPLICIT_INVERSE", str(inverse))
    import torch
    from andfn_b200 import network as nw
    from andfn_b200.adjoint import DFNModel
    F, E = nw.to_records(nw.power_law_fisher(3, nf=1500, L=30.0, ncoef=10, nint=20))
    c = _constants(10, its=500)
    model = DFNModel(F.copy(), E.copy(), c, 50)
    fr, z = _points(F, 50, 3)
    frt = torch.tensor(fr, dtype=torch.int64, device="cuda")
    zt = torch.tensor(z, dtype=torch.complex128, device="cuda")
    outlet = torch.tensor(np.nonzero((E["_type"] == 3) & (E["head"] == 0.0))[0], device="cuda")
    logt0 = np.log(F["t"].astype(np.float64))

    def J(logt, grad=False):
        lt = torch.tensor(logt, dtype=torch.float64, device="cuda", requires_grad=grad)
        coef, q, C = model.solve(lt)
        h = model.heads(coef, q, C, lt, frt, zt)
        val = (h ** 2).sum() + q[outlet].sum()
        if grad:
            val.backward()
            return lt.grad.cpu().numpy()
        return float(val)

    ga = J(logt0, grad=True)
    assert model.stats["dense_tail"] >= 256, model.stats["dense_tail"]
    assert model.adjoint_stats["status"] == 0, model.adjoint_stats
    sel = np.argsort(-np.abs(ga))[:5]
    gf = _fd(J, logt0, sel)
    err = np.abs(ga[sel] - gf)
    assert np.all(err <= 1e-5 * np.abs(ga).max()), (err / np.abs(ga).max(), ga[sel], gf)


def test_adjoint_config4_form_on_dense_tail_network():
    """The gradient check as the gradient workload states it: central finite
    differences at step 1e-6 on 20 random fractures, against both the oracle
    (the reference's algorithm on the CPU) and the GPU forward solve, with a
    per-entry relative bound of 1e-5, on the 588-fracture network whose LU
    has a 364-row dense tail.

    The 20 fractures are drawn at random among those whose gradient is at
    least 1e-3 of the largest: below that a difference quotient at step 1e-6
    is dominated by the round-off of J itself (about 3e-9 of the largest
    entry, measured), not by the gradient's error.  GPU difference quotients
    use fixed-iteration solves from the zero state (500 iterations, so J is
    smooth in log t).  The oracle's discharge solves take one refinement step
    (oracle.solve(refine=True)): the reference's unrefined SuperLU solves of
    this system (condition ~1e12) leave J noisy at ~5e-9 relative (J changes
    by 2e-11 between 150, 300 and 500 iterations, measured), which a step of
    1e-6 turns into errors of ~1e-5 of the gradient; with the refinement J is
    smooth to ~1e-15.  Its difference quotients start from its converged
    state at the base point and run 250 iterations at each perturbed point
    (the slowest mode of the iteration contracts by about 0.9 per iteration,
    so the start's influence is ~1e-11)."""
    import torch
    from andfn_b200 import network as nw
    from andfn_b200.adjoint import DFNModel
    from oracle import oracle as orc
    h = 1e-6
    F, E = nw.to_records(nw.power_law_fisher(3, nf=1500, L=30.0, ncoef=10, nint=20))
    c = _constants(10, its=500)
    model = DFNModel(F.copy(), E.copy(), c, 50)
    fr, z = _points(F, 50, 4)
    frt = torch.tensor(fr, dtype=torch.int64, device="cuda")
    zt = torch.tensor(z, dtype=torch.complex128, device="cuda")
    outlet = np.nonzero((E["_type"] == 3) & (E["head"] == 0.0))[0]
    outlet_t = torch.tensor(outlet, device="cuda")
    logt0 = np.log(F["t"].astype(np.float64))
    with torch.no_grad():
        lt = torch.tensor(logt0, dtype=torch.float64, device="cuda")
        coef, q, C = model.solve(lt)
        h0 = model.heads(coef, q, C, lt, frt, zt).cpu().numpy()
    hobs = h0 + np.random.default_rng(5).normal(0.0, 0.01, len(h0))
    hobs_t = torch.tensor(hobs, device="cuda")

    def J_gpu(logt, grad=False):
        lt = torch.tensor(logt, dtype=torch.float64, device="cuda", requires_grad=grad)
        coef, q, C = model.solve(lt)
        hh = model.heads(coef, q, C, lt, frt, zt)
        val = ((hh - hobs_t) ** 2).sum() + q[outlet_t].sum()
        if grad:
            val.backward()
            return lt.grad.cpu().numpy()
        return float(val)

    ga = J_gpu(logt0, grad=True)
    assert model.stats["dense_tail"] >= 256 and model.adjoint_stats["status"] == 0
    cand = np.nonzero(np.abs(ga) >= 1e-3 * np.abs(ga).max())[0]
    sel = np.random.default_rng(20).choice(cand, size=min(20, len(cand)), replace=False)
    assert len(sel) >= 10, len(cand)

    # the oracle: converged base state, then warm-started fixed-iteration solves
    cb = _constants(10, its=300)
    Fb, Eb = F.copy(), E.copy()
    orc.solve(Fb, Eb, 50, cb, refine=True)
    cw = _constants(10, its=250)

    def J_oracle(logt):
        Fo, Eo = Fb.copy(), Eb.copy()
        t = np.exp(logt)
        Fo["t"] = t
        m = np.isin(Eo["_type"], (2, 3))
        Eo["phi"][m] = Eo["head"][m] * t[Eo["frac0"][m]]
        orc.solve(Fo, Eo, 50, cw, refine=True)
        hh = orc.eval_heads(Fo, Eo, fr, z)
        return float(((hh - hobs) ** 2).sum() + Eo["q"][outlet].sum())

    for name, J in (("gpu", J_gpu), ("oracle", J_oracle)):
        gf = np.zeros(len(sel))
        for i, f in enumerate(sel):
            lp, lm = logt0.copy(), logt0.copy()
            lp[f] += h
            lm[f] -= h
            gf[i] = (J(lp) - J(lm)) / (2 * h)
        rel = np.abs(ga[sel] - gf) / np.abs(gf)
        print(f"adjoint vs {name} central differences (step 1e-6, {len(sel)} random fractures): "
              f"max relative {rel.max():.2e}, median {np.median(rel):.2e}")
        assert np.all(rel <= 1e-5), (name, rel, ga[sel], gf)
