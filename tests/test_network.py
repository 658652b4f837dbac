"""The numpy network generator against networks the reference itself built.

tests/golden/*.npz hold the records the reference produced from the 30-disc
recipe (andfn.Fracture + DFN.get_fracture_intersections +
set_constant_head_boundary + check_connectivity, consolidated).  The
generator must give the same fractures, the same elements in the same order
and fracture lists, and the same geometry to round-off.
"""
import numpy as np
import pytest

from andfn_b200 import network as nw
from conftest import load_golden


@pytest.mark.parametrize("case,seed", [("c1_seed3", 3), ("c1_seed13", 13), ("c1_trivial_seed0", 0)])
def test_generator_reproduces_reference_network(case, seed):
    g = load_golden(case)
    Fg, Eg = g["F_in"], g["E_in"]
    F, E = nw.to_records(nw.uniform_discs(seed), max_ncoef=Eg.dtype["coef"].shape[0],
                         max_elements=Fg.dtype["elements"].shape[0])
    assert len(F) == len(Fg) and len(E) == len(Eg)
    for name in ("_id", "_type", "frac0", "frac1", "ncoef", "nint"):
        assert np.array_equal(E[name], Eg[name]), name
    for name in ("radius", "center", "phi", "head"):
        assert np.array_equal(E[name], Eg[name]), name
    for name in ("endpoints0", "endpoints1"):
        assert np.abs(E[name] - Eg[name]).max() <= 1e-12 * max(1.0, np.abs(Eg[name]).max()), name
    assert np.array_equal(F["nelements"], Fg["nelements"])
    for f in range(len(F)):
        n = F["nelements"][f]
        assert np.array_equal(F["elements"][f, :n], Fg["elements"][f, :n])
    for name in ("t", "radius", "center"):
        assert np.array_equal(F[name], Fg[name]), name
    for name in ("normal", "x_vector", "y_vector"):
        assert np.abs(F[name] - Fg[name]).max() <= 1e-15, name


def test_power_law_recipe_spanning_cluster():
    F, E = nw.to_records(nw.power_law_fisher(5, nf=5500, L=50.0))
    assert len(F) == 2118 and len(E) == 5376
    heads = set(np.unique(E["head"][E["_type"] == 3]))
    assert heads == {0.0, 1.0}
    assert (E["_id"] == np.arange(len(E))).all() and (F["_id"] == np.arange(len(F))).all()
    # element order: bounding, impermeable circle, impermeable line, constant head, well, intersection
    order = {1: 0, 4: 1, 5: 2, 3: 3, 2: 4, 0: 5}
    assert np.all(np.diff([order[t] for t in E["_type"]]) >= 0)
