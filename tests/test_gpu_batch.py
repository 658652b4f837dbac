"""Batched realizations: every realization of a batch must give what a
separate solve of it gives.

  * against the reference's golden outputs (several networks, one batch);
  * bit-for-bit against separate GPU solves of the same networks (the batch
    runs the same per-element arithmetic in the same order; only the launch
    is shared), including iteration counts that differ between realizations;
  * against the oracle on generated networks, with realizations that stop at
    MAX_ITERATIONS (the extra sweep) beside ones that converge;
  * adaptive coefficient growth inside a batch;
  * heads of one realization through the batched handle.
Tolerances as in test_gpu_parity.
"""
import numpy as np
import pytest

from conftest import load_golden
from test_gpu_parity import _compare

pytestmark = pytest.mark.gpu


def _generated(seeds, nf=40):
    from andfn_b200 import network as nw
    return nw.to_records_batch([nw.uniform_discs(s, nf=nf, L=20.0) for s in seeds])


def _recast(a, dtype):
    """Copy of record array a in a wider dtype (same fields, larger arrays)."""
    out = np.zeros(len(a), dtype)
    for name in a.dtype.names:
        src = a[name]
        if src.ndim == 1:
            out[name] = src
        else:
            out[name][:, : src.shape[1]] = src
    return out


def test_batch_matches_reference_golden():
    import andfn_b200
    cases = ["c1_seed3", "c1_seed13", "c1_trivial_seed0", "c1_seed3"]
    gs = [load_golden(c) for c in cases]
    nets = [(g["F_in"].copy(), g["E_in"].copy()) for g in gs]
    c = gs[0]["constants_200"]
    st = andfn_b200.solve_batch(nets, 50, c)
    assert len(st) == len(cases)
    for (F, E), g, s, name in zip(nets, gs, st, cases):
        assert s["status"] in (0, 1), s
        _compare(E, F, g["E_out_200"], g["F_out_200"], ("batch", name))
    # the duplicated realization is identical to its first copy
    assert np.array_equal(nets[0][1]["coef"], nets[3][1]["coef"])


def test_batch_equals_separate_solves_bitwise(monkeypatch):
    """Every realization of a batch runs the same arithmetic as its own
    single-network solve through the triangular solves (a single network
    otherwise applies the explicit inverse of its system, a different
    summation order)."""
    monkeypatch.setenv("ANDFN_B200_EXPLICIT_INVERSE", "0")
    import andfn_b200
    from andfn_b200.records import default_constants
    recs = _generated(range(1, 9))
    c = default_constants(MAX_ITERATIONS=60, MAX_ERROR=1e-8, MAX_NCOEF=10)
    batch = [(F.copy(), E.copy()) for F, E in recs]
    st = andfn_b200.solve_batch(batch, 50, c)
    its = set()
    for (F0, E0), (Fb, Eb), s in zip(recs, batch, st):
        F, E = F0.copy(), E0.copy()
        andfn_b200.solve(F, E, 50, c)
        s1 = dict(andfn_b200.last_stats)
        assert s["iterations"] == s1["iterations"] and s["status"] == s1["status"], (s, s1)
        its.add(s["iterations"])
        for name in ("coef", "q", "error", "error_coef", "dpsi_corr", "ncoef", "nint"):
            assert np.array_equal(Eb[name], E[name], equal_nan=True), name
        assert np.array_equal(Fb["constant"], F["constant"])
    assert len(its) > 1  # realizations stopped at different iterations


def test_batch_matches_oracle_with_max_iterations_stop():
    """MAX_ITERATIONS 12: some realizations converge, the others stop at 12
    and take the reference's extra sweep (hpc_solve.py:224-234)."""
    import andfn_b200
    from andfn_b200.records import default_constants
    from oracle import oracle as orc
    g = load_golden("mixed")
    gen = _generated(range(11, 16))
    Fd, Ed = gen[0][0].dtype, gen[0][1].dtype
    assert Ed["coef"].shape[0] >= g["E_in"].dtype["coef"].shape[0]
    recs = [(_recast(g["F_in"], Fd), _recast(g["E_in"], Ed))] + gen
    c = default_constants(MAX_ITERATIONS=12, MAX_ERROR=1e-8, MAX_NCOEF=10)
    batch = [(F.copy(), E.copy()) for F, E in recs]
    st = andfn_b200.solve_batch(batch, 50, c)
    # batches solve through per-realization explicit inverses, one refinement step each solve
    assert all(s["explicit_inverse"] == 1 and s["refined_solves"] > 0 for s in st), st[0]
    for r, ((F0, E0), (Fb, Eb), s) in enumerate(zip(recs, batch, st)):
        Fo, Eo = F0.copy(), E0.copy()
        so = {}
        orc.solve(Fo, Eo, 50, c, stats=so)
        assert s["iterations"] == so["iterations"], (r, s["iterations"], so["iterations"])
        _compare(Eb, Fb, Eo, Fo, ("oracle", r))


def test_batch_adaptive_growth_matches_reference_golden():
    import andfn_b200
    g = load_golden("c1_seed3_adaptive")
    k = g["its"][-1]
    nets = [(g["F_in"].copy(), g["E_in"].copy()) for _ in range(3)]
    st = andfn_b200.solve_batch(nets, int(g["D"]), g[f"constants_{k}"])
    for (F, E), s in zip(nets, st):
        assert s["status"] in (0, 1), s
        assert (E["ncoef"] > g["E_in"]["ncoef"]).any()
        _compare(E, F, g[f"E_out_{k}"], g[f"F_out_{k}"], ("adaptive batch", int(k)))


def test_batch_handle_heads_and_rerun():
    import andfn_b200
    from andfn_b200.records import default_constants
    recs = _generated(range(21, 25))
    c = default_constants(MAX_ITERATIONS=40, MAX_ERROR=1e-8, MAX_NCOEF=10)
    batch = [(F.copy(), E.copy()) for F, E in recs]
    rng = np.random.default_rng(0)
    with andfn_b200.BatchSolver(batch, 50) as bs:
        assert bs.R == 4
        st1 = bs.run(c)
        st2 = bs.run(c)  # a second run restarts from the uploaded state
        assert [s["iterations"] for s in st1] == [s["iterations"] for s in st2]
        bs.download()
        for r, (F, E) in enumerate(batch):
            n = 500
            fr = rng.integers(0, len(F), n)
            z = F["radius"][fr] * 0.9 * np.sqrt(rng.uniform(size=n)) * np.exp(2j * np.pi * rng.uniform(size=n))
            hb = bs.eval_heads(r, fr, z)
            with andfn_b200.Solver(F, E, 50) as s:
                hs = s.eval_heads(fr, z)
            assert np.array_equal(hb, hs, equal_nan=True), r


def test_batch_realizations_with_wells_match_oracle():
    """The batched workload's own recipe (uneven sizes, the clusters touching
    a head plane, 4 wells with prescribed discharges U[-1e-4, 1e-4] on each):
    each realization vs the oracle."""
    import andfn_b200
    from andfn_b200 import network as nw
    from andfn_b200.records import default_constants
    from oracle import oracle as orc
    recs = nw.to_records_batch([nw.batch_realization(1000 + i) for i in range(8)])
    assert all(((E["_type"] == 2) & np.isnan(E["head"])).sum() == 4 for _, E in recs)
    c = default_constants(MAX_ITERATIONS=200, MAX_ERROR=1e-8, MAX_NCOEF=15)
    batch = [(F.copy(), E.copy()) for F, E in recs]
    st = andfn_b200.solve_batch(batch, 50, c)
    # batches solve through per-realization explicit inverses, one refinement step each solve
    assert all(s["explicit_inverse"] == 1 and s["refined_solves"] > 0 for s in st), st[0]
    for r, ((F0, E0), (Fb, Eb), s) in enumerate(zip(recs, batch, st)):
        Fo, Eo = F0.copy(), E0.copy()
        so = {}
        orc.solve(Fo, Eo, 50, c, stats=so)
        assert s["iterations"] == so["iterations"], (r, s["iterations"], so["iterations"])
        _compare(Eb, Fb, Eo, Fo, ("wells", r))


def test_batch_with_a_singular_realization_raises():
    """A realization whose fracture has no head boundary (one disc with a
    prescribed-discharge well only: its constant is undetermined) makes the
    batched inversion report a singular system, as the single-network path
    (SuperLU raises there, hpc_solve.py:121)."""
    import andfn_b200
    from andfn_b200 import _ffi
    from andfn_b200 import network as nw
    from andfn_b200.records import default_constants
    lone = nw.build([[0.0, 0.0, 0.0]], [[0.0, 0.0, 1.0]], [2.0], [1e-5], 10, 20, keep="all")
    nw.add_well(lone, 0, 0.3 + 0.2j, 0.05, float("nan"), q=1e-5)
    good = nw.uniform_discs(3, nf=40, L=20.0)
    recs = nw.to_records_batch([good, lone])
    c = default_constants(MAX_ITERATIONS=20, MAX_ERROR=1e-8, MAX_NCOEF=10)
    with pytest.raises(_ffi.AndfnError) as ei:
        andfn_b200.solve_batch([(F.copy(), E.copy()) for F, E in recs], 50, c)
    assert ei.value.code == 3 and "realization 1" in str(ei.value), str(ei.value)


def test_cluster_solve_of_large_realizations_is_bitwise_the_single_cta_solve(monkeypatch):
    """Realizations with at least ANDFN_B200_BINV_CLUSTER_SOLVE_N unknowns
    solve on an 8-CTA cluster each (rows split over the CTAs, x0 and the
    residual exchanged through distributed shared memory); every row's sums
    run in the same order as in the one-CTA solve, so the results are the
    same bit for bit."""
    import andfn_b200
    from andfn_b200 import network as nw
    from andfn_b200.records import default_constants
    recs = nw.to_records_batch([nw.batch_realization(2000 + i) for i in range(12)])
    c = default_constants(MAX_ITERATIONS=120, MAX_ERROR=1e-8, MAX_NCOEF=15)
    out = {}
    for thr in ("1000000", "64"):
        monkeypatch.setenv("ANDFN_B200_BINV_CLUSTER_SOLVE_N", thr)
        batch = [(F.copy(), E.copy()) for F, E in recs]
        st = andfn_b200.solve_batch(batch, 50, c)
        out[thr] = (batch, st)
    (b1, s1), (b2, s2) = out["1000000"], out["64"]
    # the clustered run launches one more kernel per iteration
    assert s2[0]["gpu_launches"] > s1[0]["gpu_launches"], (s1[0]["gpu_launches"], s2[0]["gpu_launches"])
    for r in range(len(recs)):
        assert s1[r]["iterations"] == s2[r]["iterations"] and s1[r]["status"] == s2[r]["status"], r
        for name in ("coef", "q", "error", "error_coef", "dpsi_corr", "ncoef", "nint"):
            assert np.array_equal(b1[r][1][name], b2[r][1][name], equal_nan=True), (r, name)
        assert np.array_equal(b1[r][0]["constant"], b2[r][0]["constant"]), r


def test_active_work_lists_are_bitwise_the_full_launches(monkeypatch):
    """A batch's per-iteration kernels run over lists of the running
    realizations' rows, sweep items and elements, rebuilt when one finishes;
    every entry is computed as in the full launches (where finished
    realizations return at entry), so the results are the same bit for bit,
    with realizations that stop at different iterations."""
    import andfn_b200
    from andfn_b200 import network as nw
    from andfn_b200.records import default_constants
    recs = nw.to_records_batch([nw.batch_realization(3000 + i) for i in range(16)])
    c = default_constants(MAX_ITERATIONS=120, MAX_ERROR=1e-8, MAX_NCOEF=15)
    out = {}
    for flag in ("0", "1"):
        monkeypatch.setenv("ANDFN_B200_ACTIVE_LISTS", flag)
        batch = [(F.copy(), E.copy()) for F, E in recs]
        out[flag] = (batch, andfn_b200.solve_batch(batch, 50, c))
    (b0, s0), (b1, s1) = out["0"], out["1"]
    assert len({s["iterations"] for s in s1}) > 3  # realizations finish at different iterations
    for r in range(len(recs)):
        assert s0[r]["iterations"] == s1[r]["iterations"] and s0[r]["status"] == s1[r]["status"], r
        for name in ("coef", "q", "error", "error_coef", "dpsi_corr", "ncoef", "nint"):
            assert np.array_equal(b0[r][1][name], b1[r][1][name], equal_nan=True), (r, name)
        assert np.array_equal(b0[r][0]["constant"], b1[r][0]["constant"]), r
