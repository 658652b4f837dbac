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
    from andfn_b200.fracture import calc_w
    fg, F, E, D = _load(case)
    w = calc_w(F, E, fg["w_frac"], fg["w_z"], discharge_int=D)
    ref = fg["w_ref"]
    assert np.all(np.abs(w - ref) <= TOL * np.abs(ref).max()), np.abs(w - ref).max() / np.abs(ref).max()


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


@pytest.mark.parametrize("name", ["mixed", "c1_seed3"])
def test_velocity_matches_reference_fracture_calc_velocity(name):
    """calc_velocity against the reference's own Fracture.calc_velocity: the
    velocities its streamline tracking recorded at every trace point
    (tests/golden/track_*.npz).  Left out: the last point of each segment (a
    segment that ends on an element ends on its line or circle, where w is
    singular) and the first point of each segment after a transfer (the
    reference stores the point off the intersection on the chi side there, but
    the velocity of the point the particle continues from)."""
    from andfn_b200.fracture import calc_velocity
    from test_track_golden import load_case
    t, F, E = load_case(name)
    seg = t["point_seg"]
    ends = np.cumsum(t["npoints"]) - 1
    last = np.zeros(len(seg), bool)
    last[ends[t["npoints"] > 0]] = True
    last[:-1] |= seg[1:] != seg[:-1]
    first = np.zeros(len(seg), bool)
    first[1:] = seg[1:] != seg[:-1]
    keep = ~last & ~(first & (seg > 0))
    fr, z, v_ref = t["point_frac"][keep], t["points"][keep], t["velocity"][keep]
    v = calc_velocity(F, E, fr, z, t["aperture"][fr])
    np.testing.assert_allclose(v, v_ref, rtol=1e-9, equal_nan=True)
