"""Host-side argument checks of the point-evaluation calls: the C entry
points read len(z) fracture indices and write len(z) results through the
caller's pointers, so mismatched or unsuitable arrays must be refused before
any call reaches the library (no device needed)."""
import ctypes

import numpy as np
import pytest

from andfn_b200.solver import Solver, out_array, points_args


def _unopened_solver():
    s = Solver.__new__(Solver)
    s._h = ctypes.c_void_p()
    return s


def test_points_args_converts_and_checks_lengths():
    fr, z = points_args([0, 1, 2], [0.1, 0.2j, 0.3])
    assert fr.dtype == np.int64 and z.dtype == np.complex128 and fr.shape == z.shape == (3,)
    with pytest.raises(ValueError):
        points_args([0, 1], [0.1, 0.2, 0.3])
    with pytest.raises(ValueError):
        points_args(np.zeros((2, 2), np.int64), np.zeros((2, 2), np.complex128))


@pytest.mark.parametrize("bad", [
    np.empty(5, np.float32),                       # wrong dtype
    np.empty(4),                                   # too short
    np.empty(10)[::2],                             # not contiguous
    [0.0] * 5,                                     # not an ndarray
    np.empty((5, 1)),                              # not 1-d
])
def test_out_array_refuses_unsuitable_outputs(bad):
    with pytest.raises(ValueError):
        out_array(bad, 5)


def test_out_array_refuses_read_only_and_keeps_good_arrays():
    ro = np.empty(5)
    ro.flags.writeable = False
    with pytest.raises(ValueError):
        out_array(ro, 5)
    good = np.empty(5)
    assert out_array(good, 5) is good
    assert out_array(None, 5).shape == (5,)


def test_noalloc_and_allocating_heads_refuse_bad_arguments_before_the_call():
    s = _unopened_solver()
    fr, z = np.zeros(4, np.int64), np.zeros(4, np.complex128)
    with pytest.raises(ValueError):
        s.eval_heads_noalloc(fr[:3], z)
    with pytest.raises(ValueError):
        s.eval_heads_noalloc(fr, z, out=np.empty(4, np.float32))
    with pytest.raises(ValueError):
        s.eval_heads_noalloc(fr, z, out=np.empty(3))
    with pytest.raises(ValueError):
        s.eval_heads(fr[:3], z)
    with pytest.raises(ValueError):
        s.eval_omega(fr, z[:2])
    with pytest.raises(ValueError):
        s.eval_w(fr, z[:2])
