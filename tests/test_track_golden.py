"""The streamline-tracking oracle (oracle/track.py) against traces of the
reference's own DFN.streamline_tracking (tests/golden/make_track_golden.py)."""
import os

import numpy as np
import pytest

from oracle import track as ot

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_case(name):
    t = np.load(os.path.join(HERE, f"track_{name}.npz"), allow_pickle=True)
    g = np.load(os.path.join(HERE, f"{name}.npz"), allow_pickle=True)
    k = int(t["k"])
    return t, g[f"F_out_{k}"], g[f"E_out_{k}"]


def golden_traces(t):
    """Per trace: list of (segment points, velocities, fracture)."""
    out, p = [], 0
    for n, ns in zip(t["npoints"], t["nseg"]):
        pts, vel, seg, fr = (t["points"][p:p + n], t["velocity"][p:p + n], t["point_seg"][p:p + n],
                             t["point_frac"][p:p + n])
        out.append([(pts[seg == j], vel[seg == j], int(fr[seg == j][0])) for j in range(ns)])
        p += n
    return out


def mirrors(F, E, f, z):
    """z reflected across each intersection line of fracture f (chi -> conj chi)."""
    out = []
    for k in range(int(F[f]["nelements"])):
        el = E[int(F[f]["elements"][k])]
        if int(el["_type"]) == 0:
            ep = el["endpoints0"] if f == int(el["frac0"]) else el["endpoints1"]
            out.append(ot._chi_to_z_line(np.conj(ot._line_chi(z, ep)), ep))
    return out


def assert_trace_matches(F, E, t, i, gold_i, s, sf, v, e, ztol=1e-12, vtol=1e-11, ttol=1e-12):
    """Trace i of a golden case against (segments, fractures, velocities,
    element) from an implementation.  Positions within ztol x the largest
    radius, velocities within vtol relative, travel time and length within ttol
    relative (of the golden points, with any mirrored start substituted)."""
    assert e == int(t["element"][i])
    assert len(s) == len(gold_i)
    used = []
    for j, ((gs, gv, gf), ss, vv, ff) in enumerate(zip(gold_i, s, v, sf)):
        assert ff == gf and len(ss) == len(gs)
        tol = ztol * F["radius"].max()
        if j > 0 and abs(ss[0] - gs[0]) > tol:
            # The start of a segment after a transfer is the point just off the
            # intersection on the chi side of the crossing point, which lies ON the
            # line: one rounding bit of the trace decides that side, so the mirror
            # image across an intersection of the fracture is accepted there.
            assert any(abs(ss[0] - m) <= 1e-9 * F["radius"].max() for m in mirrors(F, E, gf, gs[0]))
            gs = np.concatenate(([ss[0]], gs[1:]))
        np.testing.assert_allclose(ss, gs, rtol=0, atol=tol)
        used.append(gs)
        # A segment that ends on an element ends ON its line or circle, where w is
        # singular (the branch cut of the line map): the last rounding bit of the
        # complex square root picks the side there, so that one velocity is not
        # compared.  Travel times use v[:-1] and never read it.
        on_element = j < len(s) - 1 or e >= 0
        n = len(vv) - 1 if on_element else len(vv)
        np.testing.assert_allclose(vv[:n], gv[:n], rtol=vtol, equal_nan=True)
    tt, tl = ot.travel_time_and_length(s, v)
    np.testing.assert_allclose([tt, tl], ot.travel_time_and_length(used, [g[1] for g in gold_i]), rtol=ttol)


@pytest.mark.parametrize("name", ["mixed", "c1_seed3", "c1_seed13"])
def test_oracle_traces_match_reference(name):
    t, F, E = load_case(name)
    gold = golden_traces(t)
    for i in range(len(t["start_frac"])):
        s, sf, v, e = ot.streamline_tracking(F, E, t["aperture"], t["start_z"][i], int(t["start_frac"][i]),
                                             float(t["start_elev"][i]), float(t["ds"]), int(t["max_length"]),
                                             bool(t["backward"][i]))
        assert_trace_matches(F, E, t, i, gold[i], s, sf, v, e)
        np.testing.assert_allclose(ot.travel_time_and_length([g[0] for g in gold[i]], [g[1] for g in gold[i]]),
                                   [t["travel_time"][i], t["travel_length"][i]], rtol=1e-12)


def test_golden_cases_cover_every_exit():
    """The traces end at constant-head lines, wells, the length cap and on a
    NaN step, and several pass through intersections."""
    seen = set()
    multi = 0
    for name in ("mixed", "c1_seed3", "c1_seed13"):
        t, F, E = load_case(name)
        for e, n, ns in zip(t["element"], t["npoints"], t["nseg"]):
            seen.add(int(E["_type"][e]) if e >= 0 else (-1 if n else -2))
            multi += ns > 1
    assert {2, 3, -1, -2} <= seen and multi >= 5


def test_product_travel_time_matches_reference():
    """andfn_b200.track.get_travel_time_and_length on the reference's traces
    gives the reference's DFN.get_travel_time_and_length values."""
    from andfn_b200.track import get_travel_time_and_length
    for name in ("mixed", "c1_seed3", "c1_seed13"):
        t, F, E = load_case(name)
        for i, g in enumerate(golden_traces(t)):
            if not g:
                continue
            got = get_travel_time_and_length([x[0] for x in g], [x[1] for x in g])
            np.testing.assert_allclose(got, [t["travel_time"][i], t["travel_length"][i]], rtol=1e-14)


def test_traces_split_into_reference_segments():
    """Traces.trace turns the per-slot arrays of a launch into the reference's
    (segments, fractures, velocities, element) form, empty traces included."""
    from andfn_b200.track import Traces
    cap = 6
    z = np.arange(2 * cap, dtype=np.complex128).reshape(2, cap)
    seg = np.array([[0, 0, 1, 1, 1, 0], [0] * cap])
    fr = np.array([[3, 3, 5, 5, 5, 0], [0] * cap])
    tr = Traces(z, z.real.copy(), seg, fr, np.array([5, 0]), np.array([7, -1]), np.zeros(2, np.int32))
    s, sf, v, e = tr.trace(0)
    assert [list(x.real) for x in s] == [[0, 1], [2, 3, 4]] and sf == [3, 5] and e == 7
    assert [list(x) for x in v] == [[0, 1], [2, 3, 4]]
    assert tr.trace(1) == ([], [], [], -1)
