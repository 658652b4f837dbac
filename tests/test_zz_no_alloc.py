"""The head-evaluation entry point that allocates nothing
(andfn_b200_eval_heads_noalloc) against the allocating one, on two calls in
a row with different points, and its size limit.  Collected last so that it
also runs after every other test in the same process."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def _points(F, n, seed):
    rng = np.random.default_rng(seed)
    fr = rng.integers(0, len(F), n)
    z = F["radius"][fr] * 0.95 * np.sqrt(rng.uniform(size=n)) * np.exp(2j * np.pi * rng.uniform(size=n))
    return fr.astype(np.int64), z


def test_noalloc_heads_equal_allocating_heads_on_consecutive_calls():
    import andfn_b200
    g = load_golden("mixed")
    k = g["its"][-1]
    F, E = g[f"F_out_{k}"].copy(), g[f"E_out_{k}"].copy()
    with andfn_b200.Solver(F, E, int(g["D"])) as s:
        for seed, n in ((1, 3000), (2, 65536)):
            fr, z = _points(F, n, seed)
            h_noalloc = s.eval_heads_noalloc(fr, z)
            h_alloc = s.eval_heads(fr, z)
            assert np.array_equal(h_noalloc, h_alloc, equal_nan=True), seed


def test_noalloc_heads_after_a_solve_and_limit():
    import andfn_b200
    from andfn_b200 import _ffi
    g = load_golden("c1_seed3")
    k = g["its"][-1]
    F, E = g["F_in"].copy(), g["E_in"].copy()
    with andfn_b200.Solver(F, E, int(g["D"])) as s:
        s.run(g[f"constants_{k}"])
        fr, z = _points(F, 1000, 3)
        a = s.eval_heads_noalloc(fr, z)
        b = s.eval_heads(fr, z)
        assert np.array_equal(a, b, equal_nan=True)
        fr, z = _points(F, s.NOALLOC_MAX_POINTS + 1, 4)
        with pytest.raises(_ffi.AndfnError) as ei:
            s.eval_heads_noalloc(fr, z)
        assert ei.value.code == 11 and "65536" in str(ei.value)


def _noalloc_c(handle, fr, z, out):
    """andfn_b200_eval_heads_noalloc called through the C ABI directly."""
    import ctypes

    from andfn_b200 import _ffi
    P = ctypes.c_void_p
    return _ffi.lib().andfn_b200_eval_heads_noalloc(handle, fr.ctypes.data_as(P), z.ctypes.data_as(P), len(z),
                                                   out.ctypes.data_as(P))


def test_noalloc_heads_on_a_batch_handle_use_the_first_network():
    """On a batched handle the fracture indices are those of the first
    realization: the results equal batch_eval_heads(r=0), on two calls."""
    import andfn_b200
    gs = [load_golden("mixed"), load_golden("c1_seed3")]
    nets = []
    for g in gs:
        k = g["its"][-1]
        nets.append((g[f"F_out_{k}"].copy(), g[f"E_out_{k}"].copy()))
    with andfn_b200.BatchSolver(nets, 50) as bs:
        for seed in (5, 6):
            fr, z = _points(nets[0][0], 2000, seed)
            out = np.empty(len(z))
            assert _noalloc_c(bs._h, fr, z, out) == 0
            assert np.array_equal(out, bs.eval_heads(0, fr, z), equal_nan=True), seed


def test_noalloc_zero_points_then_a_normal_call():
    """A zero-point call (the set-up call a caller makes before capturing a
    stream) returns 0 and leaves the next call correct."""
    import andfn_b200
    g = load_golden("mixed")
    k = g["its"][-1]
    F, E = g[f"F_out_{k}"].copy(), g[f"E_out_{k}"].copy()
    with andfn_b200.Solver(F, E, int(g["D"])) as s:
        empty = np.empty(0)
        assert _noalloc_c(s._h, np.empty(0, np.int64), np.empty(0, np.complex128), empty) == 0
        fr, z = _points(F, 500, 7)
        assert np.array_equal(s.eval_heads_noalloc(fr, z), s.eval_heads(fr, z), equal_nan=True)
