"""Wells with a prescribed discharge (an extension; the reference's wells
prescribe a head): the oracle's restatement, on CPU.

Consistency: solve a network with its head-specified well to convergence,
then prescribe that well's converged discharge instead of its head; the
solution must be the same fixed point (every other unknown and every
coefficient), since the prescribed q is the value the head condition led to.
"""
import numpy as np

from conftest import load_golden, potential_scale


def _constants(its=400):
    from andfn_b200.records import default_constants
    return default_constants(MAX_ITERATIONS=its, MAX_ERROR=1e-14, MAX_NCOEF=10)


def test_prescribed_discharge_reproduces_head_specified_solution():
    from oracle import oracle as orc
    g = load_golden("mixed")
    F0, E0 = g["F_in"].copy(), g["E_in"].copy()
    wells = np.nonzero(E0["_type"] == 2)[0]
    assert len(wells) == 1
    Fh, Eh = F0.copy(), E0.copy()
    sth = {}
    orc.solve(Fh, Eh, 50, _constants(), stats=sth)
    w = wells[0]
    assert abs(Eh["q"][w]) > 0
    Fq, Eq = F0.copy(), E0.copy()
    Eq["head"][w] = np.nan
    Eq["phi"][w] = np.nan
    Eq["q"][w] = Eh["q"][w]
    stq = {}
    orc.solve(Fq, Eq, 50, _constants(), stats=stq)
    assert stq["n_unknowns"] == sth["n_unknowns"] - 1
    assert Eq["q"][w] == Eh["q"][w]  # prescribed, untouched
    P = potential_scale(Eh, Fh)
    for a, b in ((Eq["coef"], Eh["coef"]), (Eq["q"], Eh["q"]), (Fq["constant"], Fh["constant"])):
        assert np.abs(a - b).max() <= 1e-10 * P


def test_prescribed_discharge_changes_flow_linearly():
    """The solution is affine in a prescribed q: the state at q = a and at
    q = -a average to the state at q = 0."""
    from oracle import oracle as orc
    g = load_golden("mixed")
    F0, E0 = g["F_in"].copy(), g["E_in"].copy()
    w = np.nonzero(E0["_type"] == 2)[0][0]
    E0["head"][w] = np.nan
    E0["phi"][w] = np.nan
    out = []
    for qv in (1e-4, -1e-4, 0.0):
        F, E = F0.copy(), E0.copy()
        E["q"][w] = qv
        orc.solve(F, E, 50, _constants())
        out.append((E["coef"].copy(), E["q"].copy(), F["constant"].copy()))
    P = max(np.abs(out[0][0]).max(), np.abs(out[0][2]).max())
    for k in range(3):
        mid = 0.5 * (out[0][k] + out[1][k])
        assert np.abs(mid - out[2][k]).max() <= 1e-9 * P
