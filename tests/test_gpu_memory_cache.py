"""The device memory cache behind the handles' buffers: a one-call solve
gives its blocks back to the cache when its handle is destroyed, the next
call reuses them (hits, no new allocations) and gets the same results bit
for bit, and release_cached_memory() returns every block."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def test_one_call_solves_reuse_cached_blocks():
    import andfn_b200
    g = load_golden("c1_seed3")
    c = g["constants_200"]
    andfn_b200.release_cached_memory()
    assert andfn_b200.cached_memory(0)["bytes"] == 0
    outs = []
    for i in range(3):
        F, E = g["F_in"].copy(), g["E_in"].copy()
        andfn_b200.solve(F, E, 50, c)
        st = dict(andfn_b200.last_stats)
        assert st["status"] in (0, 1), st
        cm = andfn_b200.cached_memory(0)
        outs.append((F, E, cm))
        assert cm["bytes"] > 0  # the destroyed handle's blocks are kept
    # later calls are served from the cache
    assert outs[2][2]["hits"] > outs[1][2]["hits"]
    assert outs[2][2]["misses"] == outs[1][2]["misses"], (outs[1][2], outs[2][2])
    for F, E, _ in outs[1:]:
        for name in ("coef", "q", "error", "error_coef", "ncoef"):
            assert np.array_equal(E[name], outs[0][1][name], equal_nan=True), name
        assert np.array_equal(F["constant"], outs[0][0]["constant"])
    andfn_b200.release_cached_memory()
    assert andfn_b200.cached_memory(0)["bytes"] == 0

