"""Boundary-condition residual and flux balance (andfn_b200_bc_residual)
against the oracle's restatement (oracle.bc_residual) on the same solved
records: per-element residuals to rounding (the GPU evaluates the series
with FMA Horner steps, the oracle as the reference does)."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", ["c1_seed3", "mixed"])
def test_residual_of_reference_state_matches_oracle(case):
    import andfn_b200
    from oracle import oracle as orc
    g = load_golden(case)
    k = g["its"][-1]
    F, E = g[f"F_out_{k}"].copy(), g[f"E_out_{k}"].copy()
    ref = orc.bc_residual(F, E)
    with andfn_b200.Solver(F, E, int(g["D"])) as s:
        r = s.bc_residual()
    assert r["h_scale"] == ref["h_scale"] and np.isclose(r["q_scale"], ref["q_scale"], rtol=1e-14)
    assert np.allclose(r["elem"], ref["elem"], rtol=1e-6, atol=1e-11), np.abs(r["elem"] - ref["elem"]).max()
    assert np.allclose(r["flux"], ref["flux"], rtol=1e-6, atol=1e-14 * ref["q_scale"])
    assert r["bc_worst"] == int(np.argmax(ref["elem"]))


def test_residual_after_gpu_solve_matches_oracle():
    import andfn_b200
    from oracle import oracle as orc
    g = load_golden("c1_seed13")
    k = g["its"][-1]
    F, E = g["F_in"].copy(), g["E_in"].copy()
    with andfn_b200.Solver(F, E, int(g["D"])) as s:
        s.run(g[f"constants_{k}"])
        r = s.bc_residual()
        s.download()
    ref = orc.bc_residual(F, E)
    assert np.allclose(r["elem"], ref["elem"], rtol=1e-6, atol=1e-11)
    assert r["flux_max"] < 1e-10
