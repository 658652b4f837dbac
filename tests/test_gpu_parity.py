"""GPU solve against the reference's golden outputs and the pinned oracle.

Tolerances (FP64 throughout; the GPU sums in a different order and uses an
FMA-based Horner scheme, so agreement is to rounding, not bit-exact):
  * coefficients, discharges q, fracture constants, dpsi_corr:
        max |gpu - ref| <= 1e-10 * P, with P the potential scale of the
        solved network (conftest.potential_scale: max |coef|, |phi|, |C|)
  * error_coef: absolute 1e-10 * P (it is a mean |delta coef|), except where
    one side is exactly 0: calc_coef_error returns 0 when the sum of the old
    coefficients' magnitudes is below 1e-15 (hpc_math_functions.py:647-670),
    a threshold on a round-off-level sum, so an element whose old
    coefficients sit at round-off can fall on either side; such a flip is
    accepted when the nonzero value is below 1e-6 * P, for at most 0.1 % of
    the elements
  * error (the truncation indicator | |S - S_10| / |S| - 1 |, S = sum of the
    element's new coefficients): coefficient differences of 1e-10 P move it by
    at most about m 1e-10 P / |S|, so per element the bound is
    1e-7 + 1e-7 m P / |S| (|S| taken from the reference's stored coefficients,
    a margin of 1e3 over the first-order estimate)
  * ncoef, nint, thetas: exact
  * heads Re(Omega)/t at random points: |gpu - ref| <= 1e-9 * max(1, |ref|)
"""
import numpy as np
import pytest

from conftest import ADAPTIVE_CASES, GOLDEN_CASES, HEADS_CASES, load_golden, potential_scale

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _gpu_solve(F, E, D, c):
    import andfn_b200
    andfn_b200.solve(F, E, D, c)
    return dict(andfn_b200.last_stats)


def error_coef_mismatch(a, b, P):
    """Elements whose error_coef differs by more than 1e-10 P, not counting
    the threshold flips described in the module docstring; the number of
    flips."""
    d = np.abs(a - b)
    flip = ((a == 0) != (b == 0)) & (np.maximum(np.abs(a), np.abs(b)) <= 1e-6 * P)
    return np.nonzero((d > TOL * P) & ~flip)[0], int(flip.sum())


def _compare(E, F, Eo, Fo, tag):
    assert np.array_equal(E["ncoef"], Eo["ncoef"]), tag
    assert np.array_equal(E["nint"], Eo["nint"]), tag
    assert np.array_equal(E["thetas"], Eo["thetas"]), tag
    P = potential_scale(Eo, Fo)
    for name, a, b in (("coef", E["coef"], Eo["coef"]), ("q", E["q"], Eo["q"]),
                       ("constant", F["constant"], Fo["constant"]), ("dpsi_corr", E["dpsi_corr"], Eo["dpsi_corr"])):
        d = float(np.abs(a - b).max())
        assert d <= TOL * P, (tag, name, d / P)
    bad, flips = error_coef_mismatch(E["error_coef"], Eo["error_coef"], P)
    assert len(bad) == 0 and flips <= max(1, len(E) // 1000), (tag, "error_coef", bad[:5], flips)
    if P > 1e3 * max(np.abs(Eo["coef"]).max(), 1e-300):
        return  # no flow: the truncation indicator is a ratio of round-off terms
    c = Eo["coef"]
    m = np.maximum(Eo["ncoef"], 1)
    S = np.maximum(np.abs(c.sum(1)), 1e-300)
    tol = 1e-7 + 1e-7 * m * P / S
    ok = np.isfinite(Eo["error"])
    bad = np.abs(E["error"] - Eo["error"]) > tol
    assert not np.any(bad & ok), (tag, "error", np.nonzero(bad & ok)[0][:5])


@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_solve_matches_reference_golden(case):
    g = load_golden(case)
    for k in g["its"]:
        F, E = g["F_in"].copy(), g["E_in"].copy()
        st = _gpu_solve(F, E, int(g["D"]), g[f"constants_{k}"])
        assert st["status"] in (0, 1), st
        _compare(E, F, g[f"E_out_{k}"], g[f"F_out_{k}"], (case, int(k)))


@pytest.mark.parametrize("case", ADAPTIVE_CASES)
def test_adaptive_growth_matches_reference_golden(case):
    """MAX_NCOEF above ncoef: coefficients grow by COEF_INCREASE during the
    solve (element_solver2); ncoef/nint must follow the reference exactly."""
    g = load_golden(case)
    for k in g["its"]:
        F, E = g["F_in"].copy(), g["E_in"].copy()
        st = _gpu_solve(F, E, int(g["D"]), g[f"constants_{k}"])
        assert st["status"] in (0, 1), st
        assert (E["ncoef"] > g["E_in"]["ncoef"]).any() or k < 3
        _compare(E, F, g[f"E_out_{k}"], g[f"F_out_{k}"], (case, int(k)))


@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_iteration_count_matches_oracle(case):
    from oracle import oracle as orc
    g = load_golden(case)
    k = g["its"][-1]
    F, E = g["F_in"].copy(), g["E_in"].copy()
    st_o = {}
    orc.solve(F, E, int(g["D"]), g[f"constants_{k}"], stats=st_o)
    F2, E2 = g["F_in"].copy(), g["E_in"].copy()
    st = _gpu_solve(F2, E2, int(g["D"]), g[f"constants_{k}"])
    assert st["iterations"] == st_o["iterations"], (st, st_o)
    assert st["cnt_error"] == st_o["cnt_error"]


@pytest.mark.parametrize("case", HEADS_CASES)
def test_heads_match_reference(case):
    import andfn_b200
    g = load_golden(case)
    k = g["its"][-1]
    F, E = g[f"F_out_{k}"].copy(), g[f"E_out_{k}"].copy()
    with andfn_b200.Solver(F, E, int(g["D"])) as s:
        h = s.eval_heads(g["heads_frac"], g["heads_z"])
    ref = g["heads_ref"]
    assert np.all(np.abs(h - ref) <= 1e-9 * np.maximum(1.0, np.abs(ref)))


def test_heads_10k_points_after_gpu_solve():
    """Full pipeline at 10^4 points: GPU solve + GPU heads vs oracle solve +
    oracle heads on the 24-fracture network."""
    import andfn_b200
    from oracle import oracle as orc
    g = load_golden("c1_seed3")
    k = g["its"][-1]
    Fg, Eg = g["F_in"].copy(), g["E_in"].copy()
    _gpu_solve(Fg, Eg, int(g["D"]), g[f"constants_{k}"])
    Fo, Eo = g["F_in"].copy(), g["E_in"].copy()
    orc.solve(Fo, Eo, int(g["D"]), g[f"constants_{k}"])
    rng = np.random.default_rng(5)
    n = 10000
    fr = rng.integers(0, len(Fo), n)
    z = Fo["radius"][fr] * 0.95 * np.sqrt(rng.uniform(size=n)) * np.exp(2j * np.pi * rng.uniform(size=n))
    with andfn_b200.Solver(Fg, Eg, int(g["D"])) as s:
        hg = s.eval_heads(fr, z)
    ho = orc.eval_heads(Fo, Eo, fr, z)
    assert np.all(np.abs(hg - ho) <= 1e-9 * np.maximum(1.0, np.abs(ho)))


@pytest.mark.parametrize("inverse", [1, 0])
def test_generated_network_matches_oracle_with_dense_tail(inverse, monkeypatch):
    """A 551-fracture power-law/Fisher network (N = 1398 unknowns): large
    enough that the LU has a dense trailing block.  Discharge solves through
    the explicit inverse (1) or the triangular solves with dense panels (0).
    GPU vs oracle after 3 and 10 iterations."""
    monkeypatch.setenv("ANDFN_B200_EXPLICIT_INVERSE", str(inverse))
    from andfn_b200 import network as nw
    from andfn_b200.records import default_constants
    from oracle import oracle as orc
    F0, E0 = nw.to_records(nw.power_law_fisher(0, nf=1500, L=30.0, ncoef=10, nint=20))
    for its in (3, 10):
        c = default_constants(MAX_ITERATIONS=its, MAX_ERROR=1e-8, MAX_NCOEF=10)
        F, E = F0.copy(), E0.copy()
        st = _gpu_solve(F, E, 50, c)
        assert st["dense_tail"] >= 64 and st["explicit_inverse"] == inverse, st
        Fo, Eo = F0.copy(), E0.copy()
        orc.solve(Fo, Eo, 50, c)
        _compare(E, F, Eo, Fo, ("generated", its))


@pytest.mark.parametrize("inverse", [1, 0])
def test_generated_network_with_cluster_dense_tail_matches_oracle(inverse, monkeypatch):
    """A 588-fracture network with a 364-row dense tail, 120 iterations (the
    network converges at 146; a fixed count keeps the comparison exact):
    coefficients vs the oracle, with the explicit inverse of the whole system
    (1) and with the triangular solves whose dense tail runs as a CTA cluster
    (tail inverse + one refinement step) (0)."""
    monkeypatch.setenv("ANDFN_B200_EXPLICIT_INVERSE", str(inverse))
    from andfn_b200 import network as nw
    from andfn_b200.records import default_constants
    from oracle import oracle as orc
    F0, E0 = nw.to_records(nw.power_law_fisher(3, nf=1500, L=30.0, ncoef=10, nint=20))
    c = default_constants(MAX_ITERATIONS=120, MAX_ERROR=1e-300, MAX_NCOEF=10)
    F, E = F0.copy(), E0.copy()
    st = _gpu_solve(F, E, 50, c)
    assert st["dense_tail"] >= 256 and st["iterations"] == 120 and st["explicit_inverse"] == inverse, st
    if inverse:  # every explicit-inverse solve takes the refinement step
        assert st["refined_solves"] == 120, st
    Fo, Eo = F0.copy(), E0.copy()
    orc.solve(Fo, Eo, 50, c)
    _compare(E, F, Eo, Fo, ("cluster tail", 120))
