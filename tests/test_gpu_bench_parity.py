"""GPU parity on the networks the benchmark measures.

  * the plain-solve network (2,118 fractures, 5,376 elements, ncoef 20,
    nint 40): the GPU after 1 and 3 iterations and at convergence against
    the reference's own outputs (tests/golden/bench_c2.npz: full q, fracture
    constants and errors, coefficients of 256 sampled elements); the GPU
    against the oracle (pinned bit for bit to those outputs,
    test_oracle_bench_golden.py) on every coefficient after 3 and 10
    iterations and at convergence, with equal iteration counts; heads at the
    fixture's 10,000 points against the reference's heads;
  * the large network (2,588 fractures, 100 impermeable circles, ncoef 30,
    nint 60): the GPU after 1 and 2 iterations against the reference's
    outputs, and after 3 iterations against the oracle.

Tolerances (as test_gpu_parity): coefficients, q, constants, dpsi_corr and
error_coef within 1e-10 * P, P the potential scale of the network (largest
|coef|, |phi|, |constant|; error_coef with test_gpu_parity's allowance for
the reference's round-off threshold); ncoef and nint exact; heads within
1e-9 * max(1, |h|).  Each comparison also reports the per-coefficient
relative error |gpu - ref| / |ref| over the coefficients above 1e-6 P (a
coefficient far below the potential scale carries few significant digits
of the scale-sized sums it is fitted from) and requires it below 1e-6.
"""
import numpy as np
import pytest

from conftest import potential_scale
from test_gpu_parity import _compare, error_coef_mismatch
from test_oracle_bench_golden import golden_and_records

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _gpu_solve(F, E, c):
    import andfn_b200
    andfn_b200.solve(F, E, 50, c)
    return dict(andfn_b200.last_stats)


def coef_relative_error(a, b, P):
    """Largest |a - b| / |b| over the coefficients with |b| > 1e-6 P, and the
    count of such coefficients."""
    mag = np.abs(b)
    sel = mag > 1e-6 * P
    if not sel.any():
        return 0.0, 0
    return float((np.abs(a - b)[sel] / mag[sel]).max()), int(sel.sum())


def _compare_fingerprint(g, k, F, E, tag):
    """GPU state against the reference's stored outputs after k iterations."""
    p = f"k{k}_"
    s = g["sample"]
    assert np.array_equal(E["ncoef"], g[p + "ncoef"]) and np.array_equal(E["nint"], g[p + "nint"]), tag
    cs = g[p + "coef_sample"]
    P = float(max(np.abs(cs).max(), np.abs(E["phi"]).max(), np.abs(g[p + "constant"]).max()))
    for name, a, b in (("coef (sampled elements)", E["coef"][s], cs), ("q", E["q"], g[p + "q"]),
                       ("constant", F["constant"], g[p + "constant"]),
                       ("dpsi_corr (sampled elements)", E["dpsi_corr"][s], g[p + "dpsi_corr_sample"])):
        d = float(np.abs(a - b).max())
        assert d <= TOL * P, (tag, name, d / P)
    bad, flips = error_coef_mismatch(E["error_coef"], g[p + "error_coef"], P)
    if flips:
        print(f"{tag}: {flips} element(s) on the other side of calc_coef_error's 1e-15 threshold")
    assert len(bad) == 0 and flips <= max(1, len(E) // 1000), (tag, "error_coef", bad[:5], flips)
    rel, n = coef_relative_error(E["coef"][s], cs, P)
    print(f"{tag}: max |dcoef|/P {np.abs(E['coef'][s] - cs).max() / P:.2e}, per-coefficient relative {rel:.2e} "
          f"over {n} sampled coefficients")
    assert rel < 1e-6, (tag, rel)


def _compare_oracle(E, F, Eo, Fo, tag):
    _compare(E, F, Eo, Fo, tag)
    P = potential_scale(Eo, Fo)
    rel, n = coef_relative_error(E["coef"], Eo["coef"], P)
    print(f"{tag}: max |dcoef|/P {np.abs(E['coef'] - Eo['coef']).max() / P:.2e}, per-coefficient relative "
          f"{rel:.2e} over {n} coefficients")
    assert rel < 1e-6, (tag, rel)


def test_plain_network_matches_reference_outputs():
    g, F0, E0 = golden_and_records("bench_c2")
    for k in g["its"]:
        F, E = F0.copy(), E0.copy()
        st = _gpu_solve(F, E, g[f"k{k}_constants"])
        assert st["status"] in (0, 1), st
        _compare_fingerprint(g, int(k), F, E, ("bench_c2 vs reference", int(k)))


@pytest.mark.parametrize("k", [3, 10])
def test_plain_network_matches_oracle_at_fixed_iterations(k):
    from andfn_b200.records import default_constants
    from oracle import oracle as orc
    _, F0, E0 = golden_and_records("bench_c2")
    c = default_constants(MAX_ITERATIONS=k, MAX_ERROR=1e-300, MAX_NCOEF=20)
    F, E = F0.copy(), E0.copy()
    st = _gpu_solve(F, E, c)
    assert st["iterations"] == k, st
    Fo, Eo = F0.copy(), E0.copy()
    orc.solve(Fo, Eo, 50, c)
    _compare_oracle(E, F, Eo, Fo, ("bench_c2 vs oracle", k))


def test_plain_network_converges_like_the_oracle_and_heads_match_reference():
    """To convergence at MAX_ERROR 1e-8 (the benchmark's stopping rule):
    iteration counts equal, every coefficient within the bound, and heads at
    the fixture's 10,000 points against the reference's heads."""
    import andfn_b200
    from oracle import oracle as orc
    g, F0, E0 = golden_and_records("bench_c2")
    k = int(g["heads_k"])
    c = g[f"k{k}_constants"]
    F, E = F0.copy(), E0.copy()
    st = _gpu_solve(F, E, c)
    Fo, Eo = F0.copy(), E0.copy()
    sto = {}
    orc.solve(Fo, Eo, 50, c, stats=sto)
    assert st["status"] == 0 and st["iterations"] == sto["iterations"], (st, sto)
    assert st["cnt_error"] == sto["cnt_error"]
    _compare_oracle(E, F, Eo, Fo, ("bench_c2 converged vs oracle", st["iterations"]))
    with andfn_b200.Solver(F, E, 50) as s:
        h = s.eval_heads(g["heads_frac"], g["heads_z"])
    ref = g["heads_ref"]
    err = np.abs(h - ref) / np.maximum(1.0, np.abs(ref))
    print(f"bench_c2 heads at {len(ref)} points: max relative error {err.max():.2e}")
    assert np.all(err <= 1e-9)


def test_large_network_matches_reference_and_oracle():
    from andfn_b200.records import default_constants
    from oracle import oracle as orc
    g, F0, E0 = golden_and_records("bench_c5")
    assert (E0["_type"] == 4).sum() == 100
    for k in g["its"]:
        F, E = F0.copy(), E0.copy()
        st = _gpu_solve(F, E, g[f"k{k}_constants"])
        assert st["status"] in (0, 1), st
        _compare_fingerprint(g, int(k), F, E, ("bench_c5 vs reference", int(k)))
    c = default_constants(MAX_ITERATIONS=3, MAX_ERROR=1e-300, MAX_NCOEF=30)
    F, E = F0.copy(), E0.copy()
    _gpu_solve(F, E, c)
    Fo, Eo = F0.copy(), E0.copy()
    orc.solve(Fo, Eo, 50, c)
    _compare_oracle(E, F, Eo, Fo, ("bench_c5 vs oracle", 3))


@pytest.mark.parametrize("name", ["bench_c2", "bench_c5"])
def test_one_launch_dense_lu_is_bitwise_the_three_kernel_lu(name, monkeypatch):
    """The Schur complement's dense LU in one cooperative launch (look-ahead
    panel on CTA 0, bounded grid barriers) computes every product and
    quotient of the three-launch path in the same order: a solve through
    either gives the same state bit for bit."""
    from andfn_b200.records import default_constants
    _, F0, E0 = golden_and_records(name)
    mc = 20 if name == "bench_c2" else 30
    c = default_constants(MAX_ITERATIONS=3, MAX_ERROR=1e-300, MAX_NCOEF=mc)
    out = {}
    for coop in ("0", "1"):
        monkeypatch.setenv("ANDFN_B200_DLU_COOP", coop)
        F, E = F0.copy(), E0.copy()
        st = _gpu_solve(F, E, c)
        assert st["dense_tail"] >= 64, st["dense_tail"]
        out[coop] = (F, E, st)
    (F1, E1, s1), (F2, E2, s2) = out["0"], out["1"]
    assert s2["gpu_launches"] < s1["gpu_launches"]
    for field in ("coef", "q", "error", "error_coef", "dpsi_corr"):
        assert np.array_equal(E1[field], E2[field], equal_nan=True), field
    assert np.array_equal(F1["constant"], F2["constant"])


def test_single_precision_refinement_pass_matches_double(monkeypatch):
    """The refinement pass of every discharge solve reads a float copy of the
    explicit inverse (it forms the small correction X r); against both passes
    in double, on the benchmark network after 3 iterations and at
    convergence: the same iteration count and every coefficient, q and
    constant within 1e-12 of the potential scale."""
    from andfn_b200.records import default_constants
    from conftest import potential_scale
    _, F0, E0 = golden_and_records("bench_c2")
    for c in (default_constants(MAX_ITERATIONS=3, MAX_ERROR=1e-300, MAX_NCOEF=20),
              default_constants(MAX_ITERATIONS=200, MAX_ERROR=1e-8, MAX_NCOEF=20)):
        out = {}
        for flag in ("0", "1"):
            monkeypatch.setenv("ANDFN_B200_WINV_F32", flag)
            F, E = F0.copy(), E0.copy()
            st = _gpu_solve(F, E, c)
            assert st["explicit_inverse"] == 1 and st["refined_solves"] > 0, st
            out[flag] = (F, E, st)
        (F1, E1, s1), (F2, E2, s2) = out["0"], out["1"]
        assert s1["iterations"] == s2["iterations"] and s1["status"] == s2["status"]
        P = potential_scale(E1, F1)
        for name, a, b in (("coef", E1["coef"], E2["coef"]), ("q", E1["q"], E2["q"]),
                           ("constant", F1["constant"], F2["constant"])):
            d = float(np.abs(a - b).max())
            print(f"float refinement pass, {s1['iterations']} iterations: max |d {name}|/P {d / P:.2e}")
            assert d <= 1e-12 * P, (name, d / P)



def test_blocked_tail_inverse_matches_per_column_inverse(monkeypatch):
    """The dense tail's inverse W22 = U22^-1 L22^-1 formed by 64-row blocks
    (diagonal-block solves and GEMM updates) against the per-column solve:
    a different summation order, so the states after 5 and 90 iterations
    agree to round-off (1e-12 of the potential scale) with equal iteration
    counts."""
    from andfn_b200.records import default_constants
    from conftest import potential_scale
    _, F0, E0 = golden_and_records("bench_c2")
    for c in (default_constants(MAX_ITERATIONS=5, MAX_ERROR=1e-300, MAX_NCOEF=20),
              default_constants(MAX_ITERATIONS=200, MAX_ERROR=1e-8, MAX_NCOEF=20)):
        out = {}
        for flag in ("0", "1"):
            monkeypatch.setenv("ANDFN_B200_DINV_BLOCKED", flag)
            F, E = F0.copy(), E0.copy()
            st = _gpu_solve(F, E, c)
            assert st["dense_tail"] >= 64 and st["explicit_inverse"] == 1, st
            out[flag] = (F, E, st)
        (F1, E1, s1), (F2, E2, s2) = out["0"], out["1"]
        assert s1["iterations"] == s2["iterations"] and s1["status"] == s2["status"]
        P = potential_scale(E1, F1)
        for name, a, b in (("coef", E1["coef"], E2["coef"]), ("q", E1["q"], E2["q"]),
                           ("constant", F1["constant"], F2["constant"])):
            d = float(np.abs(a - b).max())
            print(f"blocked tail inverse, {s1['iterations']} iterations: max |d {name}|/P {d / P:.2e}")
            assert d <= 1e-12 * P, (name, d / P)
