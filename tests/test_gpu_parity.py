"""GPU solve against the reference's golden outputs and the pinned oracle.

Tolerances (FP64 throughout; the GPU sums in a different order and uses an
FMA-based Horner scheme, so agreement is to rounding, not bit-exact):
  * coefficients, discharges q, fracture constants, dpsi_corr:
        max |gpu - ref| <= 1e-10 * P, with P the potential scale of the
        solved network (conftest.potential_scale: max |coef|, |phi|, |C|)
  * error_coef: absolute 1e-10 * P (it is a mean |delta coef|)
  * error (the truncation indicator |  |S - S_10| / |S| - 1 |): absolute 1e-7
  * ncoef, nint, thetas: exact
  * heads Re(Omega)/t at random points: |gpu - ref| <= 1e-9 * max(1, |ref|)
"""
import numpy as np
import pytest

from conftest import GOLDEN_CASES, HEADS_CASES, load_golden, potential_scale

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _gpu_solve(F, E, D, c):
    import andfn_b200
    andfn_b200.solve(F, E, D, c)
    return dict(andfn_b200.last_stats)


def _compare(E, F, Eo, Fo, tag):
    assert np.array_equal(E["ncoef"], Eo["ncoef"]), tag
    assert np.array_equal(E["nint"], Eo["nint"]), tag
    assert np.array_equal(E["thetas"], Eo["thetas"]), tag
    P = potential_scale(Eo, Fo)
    for name, a, b in (("coef", E["coef"], Eo["coef"]), ("q", E["q"], Eo["q"]),
                       ("constant", F["constant"], Fo["constant"]), ("dpsi_corr", E["dpsi_corr"], Eo["dpsi_corr"]),
                       ("error_coef", E["error_coef"], Eo["error_coef"])):
        d = float(np.abs(a - b).max())
        assert d <= TOL * P, (tag, name, d / P)
    if P > 1e3 * max(np.abs(Eo["coef"]).max(), 1e-300):
        return  # no flow: the truncation indicator is a ratio of round-off terms
    assert np.abs(E["error"] - Eo["error"]).max() <= 1e-7, (tag, "error")


@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_solve_matches_reference_golden(case):
    g = load_golden(case)
    for k in g["its"]:
        F, E = g["F_in"].copy(), g["E_in"].copy()
        st = _gpu_solve(F, E, int(g["D"]), g[f"constants_{k}"])
        assert st["status"] in (0, 1), st
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
