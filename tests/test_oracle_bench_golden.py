"""The CPU oracle against the reference's own solve of the benchmark networks.

tests/golden/bench_*.npz were written by tests/golden/make_bench_golden.py:
the reference's andfn.hpc.hpc_solve.solve on the plain-solve network (2,118
fractures, ncoef 20, nint 40) after 1 and 3 iterations and at convergence,
and on the large network (2,588 fractures, 100 impermeable circles, ncoef 30,
nint 60) after 1 and 2 iterations.  Each output field is stored as a SHA-256
of its bytes: the oracle must reproduce every field bit for bit.  The stored
sample values say where a mismatch is when a hash differs.
"""
import hashlib

import numpy as np
import pytest

from conftest import load_golden

FIELDS = ("coef", "q", "error", "error_old", "error_old2", "error_coef", "dpsi_corr", "thetas", "ncoef", "nint")


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def records_digest(F, E):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(F).tobytes())
    h.update(np.ascontiguousarray(E).tobytes())
    return h.hexdigest()


def bench_records(name):
    """The records of a benchmark network, rebuilt from its seed exactly as
    the benchmark builds it."""
    from andfn_b200 import network as nw
    if name == "bench_c2":
        return nw.to_records(nw.power_law_fisher(5, nf=5500, L=50.0, ncoef=20, nint=40))
    if name == "bench_c5":
        return nw.to_records(nw.large_network())
    raise KeyError(name)


_cache = {}


def golden_and_records(name):
    if name not in _cache:
        g = load_golden(name)
        F, E = bench_records(name)
        assert records_digest(F, E) == str(g["input_sha"]), f"{name}: the generator built a different network"
        _cache[name] = (g, F, E)
    return _cache[name]


def check_fingerprint(g, k, F, E):
    p = f"k{k}_"
    s = g["sample"]
    diff = {}
    for name in FIELDS:
        if digest(E[name]) != str(g[p + "sha_" + name]):
            diff[name] = True
    if digest(F["constant"]) != str(g[p + "sha_constant"]):
        diff["constant"] = True
    assert not diff, (k, sorted(diff), float(np.abs(E["coef"][s] - g[p + "coef_sample"]).max()),
                      float(np.abs(E["q"] - g[p + "q"]).max()))
    # the stored values themselves (redundant with the hashes; kept readable)
    assert np.array_equal(E["coef"][s], g[p + "coef_sample"])
    assert np.array_equal(E["q"], g[p + "q"]) and np.array_equal(F["constant"], g[p + "constant"])


@pytest.mark.parametrize("name", ["bench_c2", "bench_c5"])
def test_oracle_matches_reference_on_bench_networks_bit_exact(name):
    from oracle import oracle as orc
    g, F0, E0 = golden_and_records(name)
    for k in g["its"]:
        F, E = F0.copy(), E0.copy()
        st = {}
        orc.solve(F, E, int(g["D"]), g[f"k{k}_constants"], stats=st)
        check_fingerprint(g, k, F, E)


def test_oracle_heads_match_reference_on_bench_network():
    """Heads at 10,000 seeded points of the converged plain-solve network."""
    from oracle import oracle as orc
    g, F0, E0 = golden_and_records("bench_c2")
    k = int(g["heads_k"])
    F, E = F0.copy(), E0.copy()
    orc.solve(F, E, int(g["D"]), g[f"k{k}_constants"])
    h = orc.eval_heads(F, E, g["heads_frac"], g["heads_z"])
    assert np.array_equal(h, g["heads_ref"])
