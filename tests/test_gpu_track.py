"""GPU streamline tracking (andfn_b200_track) against the reference's traces,
the oracle's object-layer field and the host-compiled copy of the same
device code."""
import numpy as np
import pytest

from andfn_b200 import Solver
from andfn_b200._ffi import AndfnError
from andfn_b200.track import calc_w_object, get_travel_time_and_length, streamline_tracking, streamlines, track
from oracle import track as ot
from test_track_golden import assert_trace_matches, golden_traces, load_case
from test_track_host import TTOL, VTOL, ZTOL, host_lib, host_track  # noqa: F401  (host_lib is a fixture)

pytestmark = pytest.mark.gpu


def solver_for(F, E):
    return Solver(np.ascontiguousarray(F), np.ascontiguousarray(E), 50)


@pytest.mark.parametrize("name", ["mixed", "c1_seed3"])
def test_gpu_tracker_matches_reference(name):
    t, F, E = load_case(name)
    gold = golden_traces(t)
    with solver_for(F, E) as s:
        for b in (False, True):
            idx = np.flatnonzero(t["backward"] == b)
            tr = track(s, t["aperture"], t["start_frac"][idx], t["start_z"][idx], t["start_elev"][idx],
                       float(t["ds"]), int(t["max_length"]), b)
            assert (tr.status == 0).all()
            for k, i in enumerate(idx):
                s_, sf, v, e = tr.trace(k)
                assert_trace_matches(F, E, t, i, gold[i], s_, sf, v, e, ZTOL, VTOL, TTOL)


@pytest.mark.parametrize("name", ["mixed", "c1_seed3"])
def test_gpu_object_w_matches_oracle(name):
    t, F, E = load_case(name)
    rng = np.random.default_rng(6)
    fr = rng.integers(0, len(F), 400)
    z = np.sqrt(rng.uniform(0, 1.0, 400)) * F["radius"][fr] * np.exp(1j * rng.uniform(0, 2 * np.pi, 400))
    with solver_for(F, E) as s:
        w = calc_w_object(F, E, fr, z, solver=s)
    ref = np.array([ot.calc_w_obj(F, E, int(f), zz) for f, zz in zip(fr, z)])
    assert np.array_equal(np.isnan(ref), np.isnan(w))
    ok = ~np.isnan(ref)
    np.testing.assert_allclose(w[ok], ref[ok], rtol=1e-10, atol=1e-12 * np.abs(ref[ok]).max())


def test_gpu_matches_host_compiled_copy(host_lib):  # noqa: F811
    """Many seeded particles, both directions: the GPU and the host-compiled
    tracker agree.  Their arithmetic differs only by fused multiply-adds, yet a
    trace can take a different discrete turn where the reference's own rules are
    ill-conditioned (a corrector that stops at |dz| = 1e-6 exactly, a step that
    grazes an element's end point); at most 3 % of the traces may do so, and
    every other trace must agree point by point."""
    t, F, E = load_case("c1_seed3")
    rng = np.random.default_rng(8)
    n = 256
    fr = rng.integers(0, len(F), n)
    z = np.sqrt(rng.uniform(0, 0.9, n)) * F["radius"][fr] * np.exp(1j * rng.uniform(0, 2 * np.pi, n))
    el = rng.uniform(0, 1, n)
    ap = t["aperture"]
    differ = 0
    with solver_for(F, E) as s:
        for b in (False, True):
            g = track(s, ap, fr, z, el, 0.01, 400, b)
            h = host_track(host_lib, F, E, ap, fr, z, el, 0.01, 400, b, 466)
            for i in range(n):
                hs, hf, hv, he = h.trace(i)
                gs, gf, gv, ge = g.trace(i)
                if ge != he or [len(x) for x in gs] != [len(x) for x in hs] or gf != hf:
                    differ += 1
                    continue
                assert_trace_matches(F, E, {"element": [he]}, 0, list(zip(hs, hv, hf)), gs, gf, gv, ge,
                                     ZTOL, VTOL, TTOL)
    assert differ <= 0.03 * 2 * n


def test_gpu_streamline_api():
    """streamline_tracking / streamlines return the reference's shapes, and the
    travel time of a trace is DFN.get_travel_time_and_length of its points."""
    t, F, E = load_case("mixed")
    f = int(t["start_frac"][1])
    z0 = t["start_z"][1]
    with solver_for(F, E) as s:
        seg, sf, v, e = streamline_tracking(F, E, z0, f, float(t["start_elev"][1]), float(t["ds"]),
                                            int(t["max_length"]), False, aperture=t["aperture"], solver=s)
        lines, fracs, vels, elems, l3 = streamlines(F, E, [z0, 0.5 * z0], f, float(t["ds"]), int(t["max_length"]),
                                                    [0.25, 0.75], remove_false=False, aperture=t["aperture"],
                                                    solver=s)
    assert len(seg) == len(sf) == len(v) and all(len(a) == len(b) for a, b in zip(seg, v))
    assert len(lines) == len(fracs) == len(vels) == len(elems) == 4
    assert all(p.ndim == 2 and p.shape[1] == 3 for p in l3)
    np.testing.assert_allclose(get_travel_time_and_length(seg, v), ot.travel_time_and_length(seg, v), rtol=1e-14)


def test_gpu_track_rejects_bad_input():
    t, F, E = load_case("mixed")
    with solver_for(F, E) as s:
        with pytest.raises(AndfnError):
            track(s, t["aperture"], [len(F)], [0.0j], [0.5], 0.01, 10)
        with pytest.raises(AndfnError):
            track(s, t["aperture"], [0], [0.0j], [0.5], 0.01, 10, cap=1)
