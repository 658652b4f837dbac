"""The CPU oracle against golden vectors written by the reference itself.

tests/golden/*.npz were produced by tests/golden/make_golden.py running the
reference's andfn.hpc.hpc_solve.solve.  The oracle restates that solver with
Numba's complex arithmetic and SciPy's SuperLU, so it must reproduce the
golden outputs exactly (bit for bit) -- this pins the oracle that every GPU
parity test is checked against.
"""
import numpy as np
import pytest

from conftest import ADAPTIVE_CASES, GOLDEN_CASES, HEADS_CASES, load_golden
from oracle import oracle as orc

FIELDS_F = ("coef", "q", "error", "error_old", "error_old2", "error_coef", "dpsi_corr", "thetas")
FIELDS_I = ("ncoef", "nint")


@pytest.mark.parametrize("case", GOLDEN_CASES + ADAPTIVE_CASES)
def test_oracle_matches_reference_bit_exact(case):
    g = load_golden(case)
    for k in g["its"]:
        F, E = g["F_in"].copy(), g["E_in"].copy()
        orc.solve(F, E, int(g["D"]), g[f"constants_{k}"])
        Eo, Fo = g[f"E_out_{k}"], g[f"F_out_{k}"]
        for name in FIELDS_I:
            assert np.array_equal(E[name], Eo[name]), (case, k, name)
        for name in FIELDS_F:
            assert np.array_equal(E[name], Eo[name], equal_nan=True), (case, k, name, np.abs(E[name] - Eo[name]).max())
        assert np.array_equal(F["constant"], Fo["constant"]), (case, k)


@pytest.mark.parametrize("case", HEADS_CASES)
def test_oracle_heads_match_reference(case):
    g = load_golden(case)
    k = g["its"][-1]
    h = orc.eval_heads(g[f"F_out_{k}"], g[f"E_out_{k}"], g["heads_frac"], g["heads_z"])
    assert np.array_equal(h, g["heads_ref"])


def test_oracle_layout_independent():
    """Same solve with the reference's default record capacity (MAX_NCOEF=200,
    MAX_ELEMENTS=500) as with the compact records of the fixture."""
    from andfn_b200.records import element_dtype, fracture_dtype
    g = load_golden("c1_seed3")
    k = 5

    def widen(a, dt):
        out = np.zeros(len(a), dt)
        for n in dt.names:
            if a[n].ndim == 1:
                out[n] = a[n]
            else:
                out[n][:, : a[n].shape[1]] = a[n]
        return out
    F = widen(g["F_in"], fracture_dtype(500))
    E = widen(g["E_in"], element_dtype(200))
    assert E.dtype.itemsize == 12992 and F.dtype.itemsize == 4136
    orc.solve(F, E, int(g["D"]), g[f"constants_{k}"])
    m = g["E_out_5"]["coef"].shape[1]
    assert np.array_equal(E["coef"][:, :m], g["E_out_5"]["coef"])
