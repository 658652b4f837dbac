"""Network geometry on the GPU (andfn_b200_disc_intersections,
andfn_b200_clusters) against the host restatement (andfn_b200/network.py,
which reproduces the reference's get_fracture_intersections and
check_connectivity element for element, tests/test_network.py).

The device rounds every operation on its own in numpy's order, so the
intersection segments must be equal bit for bit, and the networks the two
paths build -- and their solve records -- identical."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _segments(net):
    return [(e.frac0, e.frac1, e.ep0, e.ep1) for e in net.elements if e.type == 0]


@pytest.mark.parametrize("recipe", ["plain", "large"])
def test_gpu_intersections_equal_host_bit_for_bit(recipe):
    from andfn_b200 import network as nw
    if recipe == "plain":
        kw = dict(seed=5, nf=5500, L=50.0, ncoef=20, nint=40)
    else:
        kw = dict(seed=11, nf=20000, L=200.0, rmin=1.0, rmax=40.0, ncoef=30, nint=60)
    host = nw.power_law_fisher(keep="all", **kw)
    dev = nw.power_law_fisher(keep="all", device=0, **kw)
    sh, sd = _segments(host), _segments(dev)
    assert len(sh) == len(sd) > 0
    for a, b in zip(sh, sd):
        assert a[:2] == b[:2]
        assert np.array_equal(np.array(a[2] + a[3]), np.array(b[2] + b[3])), (a, b)
    # clusters of the whole set: the same labels (smallest index of each component)
    assert np.array_equal(nw._clusters(host), nw._clusters(dev, device=0))


def test_gpu_built_network_gives_the_benchmark_records():
    """The plain-solve network built with the GPU steps has the records whose
    hash the reference's own solve was pinned on."""
    from andfn_b200 import network as nw
    from conftest import load_golden
    from test_oracle_bench_golden import records_digest
    F, E = nw.to_records(nw.power_law_fisher(5, nf=5500, L=50.0, ncoef=20, nint=40, device=0))
    assert records_digest(F, E) == str(load_golden("bench_c2")["input_sha"])


def test_gpu_clusters_of_a_small_graph():
    from andfn_b200 import network as nw
    pairs = np.array([[0, 3], [3, 5], [1, 2], [6, 7], [5, 7]])
    lab = nw.gpu_clusters(9, pairs, 0)
    assert lab.tolist() == [0, 1, 1, 0, 4, 0, 0, 0, 8]
