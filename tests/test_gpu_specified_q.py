"""Wells with a prescribed discharge on the GPU (an extension; the reference's
wells prescribe a head): against the oracle's restatement
(tests/test_specified_q_oracle.py checks that restatement on CPU).

A NaN head marks such a well; its record's q is the prescribed discharge.
Its row and column leave the discharge system and its known terms move to
the right-hand side.  Tolerances as test_gpu_parity.
"""
import numpy as np
import pytest

from conftest import load_golden
from test_gpu_parity import _compare

pytestmark = pytest.mark.gpu


def _mixed_with_prescribed_well(q=7.5e-5):
    g = load_golden("mixed")
    F, E = g["F_in"].copy(), g["E_in"].copy()
    w = np.nonzero(E["_type"] == 2)[0][0]
    E["head"][w] = np.nan
    E["phi"][w] = np.nan
    E["q"][w] = q
    return F, E, w


@pytest.mark.parametrize("its", [3, 200])
def test_prescribed_discharge_well_matches_oracle(its):
    import andfn_b200
    from andfn_b200.records import default_constants
    from oracle import oracle as orc
    F0, E0, w = _mixed_with_prescribed_well()
    c = default_constants(MAX_ITERATIONS=its, MAX_ERROR=1e-8, MAX_NCOEF=10)
    F, E = F0.copy(), E0.copy()
    andfn_b200.solve(F, E, 50, c)
    st = dict(andfn_b200.last_stats)
    Fo, Eo = F0.copy(), E0.copy()
    so = {}
    orc.solve(Fo, Eo, 50, c, stats=so)
    assert st["n_unknowns"] == so["n_unknowns"] and st["iterations"] == so["iterations"], (st, so)
    assert E["q"][w] == E0["q"][w]
    _compare(E, F, Eo, Fo, ("prescribed q", its))


def test_adjoint_refuses_prescribed_discharge_wells():
    from andfn_b200 import _ffi
    from andfn_b200.adjoint import DFNModel
    from andfn_b200.records import default_constants
    import torch
    F, E, _ = _mixed_with_prescribed_well()
    c = default_constants(MAX_ITERATIONS=50, MAX_ERROR=1e-8, MAX_NCOEF=10)
    m = DFNModel(F.copy(), E.copy(), c, 50)
    lt = torch.tensor(np.log(F["t"]), dtype=torch.float64, device="cuda", requires_grad=True)
    coef, q, C = m.solve(lt)
    with pytest.raises(_ffi.AndfnError):
        q.sum().backward()
    m.close()
