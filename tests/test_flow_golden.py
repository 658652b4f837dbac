"""Flow-field restatements against the reference's own outputs (CPU): the
sunflower points and their 3-D mapping of the library's Python layer, and the
oracle's complex discharge vector, against tests/golden/flow_*.npz (written
by tests/golden/make_flow_golden.py from andfn/hpc/hpc_fracture.py)."""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = ["mixed", "c1_seed3"]


def _load(case):
    fg = np.load(os.path.join(HERE, "golden", f"flow_{case}.npz"))
    g = np.load(os.path.join(HERE, "golden", f"{case}.npz"), allow_pickle=True)
    k = int(fg["k"])
    return fg, g[f"F_out_{k}"].copy(), g[f"E_out_{k}"].copy()


@pytest.mark.parametrize("case", CASES)
def test_sunflower_points_and_3d_mapping_match_reference(case):
    from andfn_b200.fracture import map_2d_to_3d, sunflower_spiral
    from oracle import oracle as orc
    fg, F, E = _load(case)
    n = len(fg["spiral"])
    s = sunflower_spiral(n - 12, 12)
    assert np.array_equal(s, fg["spiral"])
    assert np.array_equal(orc.sunflower_spiral(n - 12, 12), fg["spiral"])
    z = s[None, :] * F["radius"][:, None]
    assert np.allclose(map_2d_to_3d(F, z), fg["flow_pnts"], rtol=0, atol=1e-12)
    assert np.allclose(map_2d_to_3d(F, z), fg["grid_pnts"], rtol=0, atol=1e-12)


@pytest.mark.parametrize("case", CASES)
def test_oracle_discharge_vector_matches_reference(case):
    from oracle import oracle as orc
    fg, F, E = _load(case)
    w = np.array([orc.calc_w(F, E, int(f), z) for f, z in zip(fg["w_frac"], fg["w_z"])])
    ref = fg["w_ref"]
    assert np.all(np.abs(w - ref) <= 1e-13 * np.abs(ref).max())
