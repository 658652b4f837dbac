"""Host factorisation (CPU): the deferred dense block.  For one network the
library stops the host LU after the Schur complement, factorises it on the
GPU and completes the factors from the pivots and U's diagonal
(sparse_lu_finish).  Here a C++ driver (tests/native/lu_defer_check.cpp)
factorises the Schur complement with the same pivot rule on the CPU and
checks that the completed factors equal the host's own factorisation."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT


def test_deferred_dense_block_matches_host_factorisation(tmp_path):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no C++ compiler")
    from andfn_b200 import network as nw
    from oracle import oracle as orc
    exe = tmp_path / "lu_defer_check"
    csrc = os.path.join(ROOT, "andfn_b200", "csrc")
    subprocess.run([gxx, "-O2", "-std=c++17", "-fopenmp", "-I", csrc,
                    os.path.join(ROOT, "tests", "native", "lu_defer_check.cpp"),
                    os.path.join(csrc, "sparse_lu.cpp"), "-o", str(exe)], check=True)
    F, E = nw.to_records(nw.power_law_fisher(0, nf=1500, L=30.0, ncoef=10, nint=20))
    A = orc.Oracle(F, E, 50).build_matrix().tocsc()
    A.sum_duplicates()
    A.sort_indices()
    parts = [f"{A.shape[0]} {A.nnz}", " ".join(map(str, A.indptr)), " ".join(map(str, A.indices)),
             " ".join(repr(float(v)) for v in A.data)]
    r = subprocess.run([str(exe)], input="\n".join(parts), capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.startswith("ok"), (r.returncode, r.stdout, r.stderr)
    assert int(r.stdout.split()[2]) >= 64


def test_leading_steps_following_the_ordering_give_the_same_factors(tmp_path):
    """A one-call solve publishes the column order while it is computed and
    takes the leading sparse pivot steps as the columns arrive
    (tests/native/lu_follow_check.cpp): the order, the dense tail and the
    factors, deferred and not, equal the sequential path's bit for bit."""
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no C++ compiler")
    from andfn_b200 import network as nw
    from oracle import oracle as orc
    exe = tmp_path / "lu_follow_check"
    csrc = os.path.join(ROOT, "andfn_b200", "csrc")
    subprocess.run([gxx, "-O2", "-std=c++17", "-fopenmp", "-pthread", "-I", csrc,
                    os.path.join(ROOT, "tests", "native", "lu_follow_check.cpp"),
                    os.path.join(csrc, "sparse_lu.cpp"), "-o", str(exe)], check=True)
    F, E = nw.to_records(nw.power_law_fisher(0, nf=1500, L=30.0, ncoef=10, nint=20))
    A = orc.Oracle(F, E, 50).build_matrix().tocsc()
    A.sum_duplicates()
    A.sort_indices()
    parts = [f"{A.shape[0]} {A.nnz}", " ".join(map(str, A.indptr)), " ".join(map(str, A.indices)),
             " ".join(repr(float(v)) for v in A.data)]
    r = subprocess.run([str(exe)], input="\n".join(parts), capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.startswith("ok"), (r.returncode, r.stdout, r.stderr)
    assert int(r.stdout.split()[1]) >= 64
