import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def load_golden(name):
    with np.load(os.path.join(GOLDEN, f"{name}.npz"), allow_pickle=False) as z:
        return {k: z[k] for k in z.files}


GOLDEN_CASES = ["c1_seed3", "c1_seed13", "c1_trivial_seed0", "mixed"]
ADAPTIVE_CASES = ["c1_seed3_adaptive"]
HEADS_CASES = ["c1_seed3", "mixed"]


@pytest.fixture(scope="session")
def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def rel_err(a, b, scale=None):
    a = np.asarray(a)
    b = np.asarray(b)
    s = np.max(np.abs(b)) if scale is None else scale
    if s == 0:
        return float(np.max(np.abs(a - b)))
    return float(np.max(np.abs(a - b)) / s)


def potential_scale(E, F):
    """Scale of the discharge potential of a solved network: the largest of
    |coef|, |phi| of head-specified elements and |fracture constant|.  Errors
    of coefficients, discharges and constants are measured against it (a
    network without flow has coefficients at round-off level, so their own
    maximum is no scale)."""
    return float(max(np.abs(E["coef"]).max(), np.abs(E["phi"]).max(), np.abs(F["constant"]).max()))
