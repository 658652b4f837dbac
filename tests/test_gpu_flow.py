"""Flow fields on the GPU against the reference's own outputs: the complex
discharge vector calc_w at random points, the flow nets (Omega at the
sunflower points of every fracture, returned with the reference's [nf, n, n]
shape) and head grids, for a converged network with every element type and a
30-disc network (tests/golden/flow_*.npz)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = ["mixed", "c1_seed3"]
TOL = 1e-10


def _load(case):
    fg = np.load(os.path.join(HERE, "golden", f"flow_{case}.npz"))
    g = np.load(os.path.join(HERE, "golden", f"{case}.npz"), allow_pickle=True)
    k = int(fg["k"])
    return fg, g[f"F_out_{k}"].copy(), g[f"E_out_{k}"].copy(), int(g["D"])


@pytest.mark.parametrize("case", CASES)
def test_discharge_vector_matches_reference(case):
    from andfn_b200.fracture import calc_velocity, calc_w
    fg, F, E, D = _load(case)
    w = calc_w(F, E, fg["w_frac"], fg["w_z"], discharge_int=D)
    ref = fg["w_ref"]
    assert np.all(np.abs(w - ref) <= TOL * np.abs(ref).max()), np.abs(w - ref).max() / np.abs(ref).max()
    v = calc_velocity(F, E, fg["w_frac"], fg["w_z"], 1e-3, discharge_int=D)
    assert np.allclose(v, np.abs(ref) / 1e-3, rtol=1e-9, atol=0)


@pytest.mark.parametrize("case", CASES)
def test_flow_nets_and_head_grid_match_reference(case):
    import andfn_b200
    from andfn_b200.fracture import get_flow_nets, get_heads
    fg, F, E, D = _load(case)
    n = len(fg["spiral"])
    with andfn_b200.Solver(F, E, D) as s:  # one upload for both
        nets, pnts = get_flow_nets(F, n - 12, 12, E, solver=s)
        heads, hp = get_heads(F, E, fg["spiral"], solver=s)
    ref = fg["flow_omega"]
    assert nets.shape == (len(F), n, n) and np.array_equal(nets[:, :, 0], nets[:, :, -1], equal_nan=True)
    om = nets[:, :, 0]
    assert np.array_equal(np.isnan(om), np.isnan(ref))
    ok = ~np.isnan(ref)
    scale = max(1.0, np.abs(ref[ok]).max())
    assert np.all(np.abs(om[ok] - ref[ok]) <= TOL * scale)
    assert np.allclose(pnts, fg["flow_pnts"], rtol=0, atol=1e-12)
    href = fg["grid_heads"]
    assert np.array_equal(np.isnan(heads), np.isnan(href))
    okh = ~np.isnan(href)
    assert np.all(np.abs(heads[okh] - href[okh]) <= 1e-9 * np.maximum(1.0, np.abs(href[okh])))
