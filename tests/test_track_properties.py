"""The tracker's device code (compiled for the host) on fresh seeded particles:
against the oracle's tracker, and invariants every trace must satisfy."""
import numpy as np
import pytest

from oracle import track as ot
from test_track_golden import assert_trace_matches, load_case
from test_track_host import TTOL, VTOL, ZTOL, host_lib, host_track  # noqa: F401  (host_lib is a fixture)


def seeded_particles(F, n, seed):
    rng = np.random.default_rng(seed)
    fr = rng.integers(0, len(F), n)
    z = np.sqrt(rng.uniform(0, 0.95, n)) * F["radius"][fr] * np.exp(1j * rng.uniform(0, 2 * np.pi, n))
    return fr, z, rng.uniform(0, 1, n)


@pytest.mark.parametrize("name,backward", [("mixed", False), ("mixed", True), ("c1_seed3", False),
                                           ("c1_seed3", True)])
def test_host_tracker_matches_oracle_on_fresh_particles(host_lib, name, backward):  # noqa: F811
    t, F, E = load_case(name)
    fr, z, el = seeded_particles(F, 10, 31 + backward)
    ap = t["aperture"]
    h = host_track(host_lib, F, E, ap, fr, z, el, 0.01, 250, backward, 316)
    for i in range(len(fr)):
        s, sf, v, e = ot.streamline_tracking(F, E, ap, z[i], int(fr[i]), float(el[i]), 0.01, 250, backward)
        gold = list(zip(s, v, sf))
        hs, hf, hv, he = h.trace(i)
        assert_trace_matches(F, E, {"element": [e]}, 0, gold, hs, hf, hv, he, ZTOL, VTOL, TTOL)


def test_trace_invariants(host_lib):  # noqa: F811
    """On 300 particles in each direction: consecutive segments are on the two
    fractures of an intersection; every point lies in its fracture's disc (up
    to the 1e-4 chi offset off an intersection's end); a trace ending on a
    constant-head line ends on that line; travel times are positive."""
    t, F, E = load_case("c1_seed3")
    ap = t["aperture"]
    fr, z, el = seeded_particles(F, 300, 41)
    pairs = {(int(a), int(b)) for a, b, ty in zip(E["frac0"], E["frac1"], E["_type"]) if ty == 0}
    pairs |= {(b, a) for a, b in pairs}
    n_transfer = n_ch = 0
    for backward in (False, True):
        h = host_track(host_lib, F, E, ap, fr, z, el, 0.01, 300, backward, 366)
        assert (h.status == 0).all()
        for i in range(len(fr)):
            s, sf, v, e = h.trace(i)
            for a, b in zip(sf[:-1], sf[1:]):
                assert (a, b) in pairs
                n_transfer += 1
            for seg, f in zip(s, sf):
                assert np.all(np.abs(seg) <= F["radius"][f] * (1 + 1e-3))
            if e >= 0 and E["_type"][e] == 3:
                n_ch += 1
                a_, b_ = E["endpoints0"][e]
                zl = s[-1][-1]
                assert abs(abs(zl - a_) + abs(zl - b_) - abs(b_ - a_)) < 1e-9 * F["radius"].max()
            if s and len(s[0]) > 1 and np.all(np.isfinite(np.concatenate(v)[:-1])):
                tt, tl = ot.travel_time_and_length(s, v)
                assert tt > 0 and tl > 0
    assert n_transfer > 20 and n_ch > 5
