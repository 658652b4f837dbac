"""The tracker's device code (andfn_b200/csrc/track.cuh) compiled for the host
(tests/native/track_host_check.cu) against the reference's traces and the
oracle's object-layer field.  The GPU runs these same functions in
track_kernel; this checks their logic and arithmetic without a GPU."""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

from andfn_b200.track import Traces
from oracle import track as ot
from test_track_golden import assert_trace_matches, golden_traces, load_case

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# Tolerances of an implementation that divides by Smith's quotient everywhere
# (the reference divides some quotients with NumPy's algorithm) -- a few ulps
# per step, over hundreds of steps.
ZTOL, VTOL, TTOL = 1e-10, 1e-9, 1e-9


@pytest.fixture(scope="module")
def host_lib(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc) and not shutil.which("nvcc"):
        pytest.skip("nvcc not available")
    out = tmp_path_factory.mktemp("track") / "track_host.so"
    subprocess.run([nvcc, "-O2", "-std=c++17", "-Wno-deprecated-gpu-targets", "-Xcompiler", "-fPIC", "-shared", "-I",
                    os.path.join(ROOT, "andfn_b200", "csrc"), "-o", str(out),
                    os.path.join(ROOT, "tests", "native", "track_host_check.cu")], check=True, timeout=600)
    return ctypes.CDLL(str(out))


def view_arrays(F, E, aperture):
    """The TrackView arrays the library builds on the device, from records."""
    ne, MC = len(E), E["coef"].shape[1]
    fptr = np.zeros(len(F) + 1, np.int32)
    felem = []
    for f in range(len(F)):
        n = int(F["nelements"][f])
        felem.extend(int(x) for x in F["elements"][f][:n])
        fptr[f + 1] = len(felem)
    geo = np.concatenate([F["radius"][:, None], F["center"], F["x_vector"], F["y_vector"], F["normal"]], axis=1)
    arrs = [np.ascontiguousarray(E["_type"], np.int32), np.ascontiguousarray(E["frac0"], np.int32),
            np.ascontiguousarray(E["frac1"], np.int32), np.ascontiguousarray(E["ncoef"], np.int32),
            np.ascontiguousarray(E["endpoints0"], np.complex128), np.ascontiguousarray(E["endpoints1"], np.complex128),
            np.ascontiguousarray(E["radius"], np.float64), np.ascontiguousarray(E["center"], np.complex128),
            np.ascontiguousarray(E["q"], np.float64), np.ascontiguousarray(E["coef"], np.complex128).reshape(ne, MC),
            fptr, np.asarray(felem, np.int32), np.ascontiguousarray(geo, np.float64),
            np.ascontiguousarray(np.broadcast_to(np.asarray(aperture, np.float64), (len(F),)))]
    return MC, arrs


def P(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def host_track(lib, F, E, aperture, frac, z0, elev, ds, max_length, backward, cap):
    MC, arrs = view_arrays(F, E, aperture)
    n = len(z0)
    frac = np.ascontiguousarray(frac, np.int32)
    z0 = np.ascontiguousarray(z0, np.complex128)
    elev = np.ascontiguousarray(elev, np.float64)
    oz = np.zeros((n, cap), np.complex128)
    ov = np.zeros((n, cap))
    oseg = np.zeros((n, cap), np.int32)
    ofr = np.zeros((n, cap), np.int32)
    on, oel, ost = np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros(n, np.int32)
    lib.track_host(ctypes.c_int(MC), *[P(a) for a in arrs], ctypes.c_int(n), P(frac), P(z0), P(elev),
                   ctypes.c_double(ds), ctypes.c_int(max_length), ctypes.c_int(int(backward)), ctypes.c_int(cap),
                   P(oz), P(ov), P(oseg), P(ofr), P(on), P(oel), P(ost))
    return Traces(oz, ov, oseg.astype(np.int64), ofr.astype(np.int64), on.astype(np.int64), oel.astype(np.int64),
                  ost)


@pytest.mark.parametrize("name", ["mixed", "c1_seed3", "c1_seed13"])
def test_host_compiled_tracker_matches_reference(host_lib, name):
    t, F, E = load_case(name)
    gold = golden_traces(t)
    for b in (False, True):
        idx = np.flatnonzero(t["backward"] == b)
        tr = host_track(host_lib, F, E, t["aperture"], t["start_frac"][idx], t["start_z"][idx],
                        t["start_elev"][idx], float(t["ds"]), int(t["max_length"]), b, int(t["max_length"]) + 66)
        assert (tr.status == 0).all()
        for k, i in enumerate(idx):
            s, sf, v, e = tr.trace(k)
            assert_trace_matches(F, E, t, i, gold[i], s, sf, v, e, ZTOL, VTOL, TTOL)


@pytest.mark.parametrize("name", ["mixed", "c1_seed3"])
def test_host_compiled_object_w_matches_oracle(host_lib, name):
    t, F, E = load_case(name)
    rng = np.random.default_rng(5)
    fr = rng.integers(0, len(F), 300)
    z = np.sqrt(rng.uniform(0, 1.0, 300)) * F["radius"][fr] * np.exp(1j * rng.uniform(0, 2 * np.pi, 300))
    MC, arrs = view_arrays(F, E, 1.0)
    out = np.zeros(300, np.complex128)
    fr32 = fr.astype(np.int32)
    host_lib.w_object_host(ctypes.c_int(MC), *[P(a) for a in arrs], ctypes.c_int(300), P(fr32), P(z), P(out))
    ref = np.array([ot.calc_w_obj(F, E, int(f), zz) for f, zz in zip(fr, z)])
    assert np.isnan(ref).sum() == np.isnan(out).sum()
    ok = ~np.isnan(ref)
    np.testing.assert_allclose(out[ok], ref[ok], rtol=1e-10, atol=1e-12 * np.abs(ref[ok]).max())


def test_truncation_at_cap(host_lib):
    """A cap smaller than the trace stops it with TRACK_TRUNCATED, every
    written point inside the slots."""
    t, F, E = load_case("c1_seed3")
    i = int(np.argmax(t["npoints"]))
    tr = host_track(host_lib, F, E, t["aperture"], t["start_frac"][[i]], t["start_z"][[i]], t["start_elev"][[i]],
                    float(t["ds"]), int(t["max_length"]), bool(t["backward"][i]), 20)
    assert tr.status[0] == 1 and tr.npoints[0] == 20 and tr.element[0] == -1
