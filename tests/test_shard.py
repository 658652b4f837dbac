"""Batched realizations split across ranks (andfn_b200.shard), on CPU.

The partition is checked directly; the sharded solve runs on two gloo ranks
with the oracle as the per-rank solver (the GPU batch solve is the default
solver on a GPU machine; the partition, the in-place updates and the
statistics gather are the same code either way).  Every realization's
statistics and records must equal those of a single-rank solve of the whole
batch.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from andfn_b200.shard import partition_lpt, sweep_pairs
from conftest import load_golden


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_partition_covers_every_realization_once_and_balances():
    rng = np.random.default_rng(0)
    w = rng.integers(100, 1000, 256).astype(float)
    for ws in (1, 2, 3, 8):
        parts = partition_lpt(w, ws)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(w)))
        loads = [w[p].sum() for p in parts]
        # LPT: the largest load exceeds the mean by less than the largest weight
        assert max(loads) - w.sum() / ws < w.max()
        assert parts == partition_lpt(w, ws)  # deterministic
    # a small case worked by hand: 5 -> r0, 4 -> r1, 3 -> r1, 3 -> r0, 3 -> r1
    # (loads 8 and 10; LPT's 4/3 bound against the optimum of 9)
    assert partition_lpt([5, 4, 3, 3, 3], 2) == [[0, 3], [1, 2, 4]]


def test_sweep_pairs_counts_point_source_pairs():
    g = load_golden("mixed")
    F, E = g["F_in"], g["E_in"]
    n = 0
    for e in range(len(E)):
        if E["_type"][e] == 2:
            continue
        sides = [E["frac0"][e]] + ([E["frac1"][e]] if E["_type"][e] == 0 else [])
        for f in sides:
            n += E["nint"][e] * F["nelements"][f]
    assert sweep_pairs(F, E) == n


def _networks():
    from andfn_b200 import network as nw
    nets = [(load_golden(c)["F_in"].copy(), load_golden(c)["E_in"].copy()) for c in ("c1_seed3", "c1_seed13")]
    nets += [nw.to_records(nw.uniform_discs(s, nf=40, L=20.0)) for s in (1, 2, 3)]
    return nets


def _constants():
    from andfn_b200.records import default_constants
    return default_constants(MAX_ITERATIONS=60, MAX_ERROR=1e-8, MAX_NCOEF=10)


def oracle_solver(share, D, c):
    from oracle import oracle as orc
    out = []
    for F, E in share:
        st = {}
        orc.solve(F, E, D, c, stats=st)
        out.append({k: st[k] for k in ("iterations", "cnt_error", "error", "error_coef")})
    return out


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    from andfn_b200.shard import solve_batch_sharded
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    nets = _networks()
    stats = solve_batch_sharded(nets, 50, _constants(), solve_fn=oracle_solver)
    parts = partition_lpt([sweep_pairs(F, E) for F, E in nets], world)
    out[rank] = (stats, {i: nets[i][1]["coef"].copy() for i in parts[rank]})
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_batch_equals_single_rank_batch():
    nets = _networks()
    ref = oracle_solver(nets, 50, _constants())
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
        res = dict(out)
    seen = set()
    for r in (0, 1):
        stats, coefs = res[r]
        assert stats == ref  # every rank holds every realization's statistics, in order
        for i, c in coefs.items():
            assert np.array_equal(c, nets[i][1]["coef"])  # this rank's share was solved in place
            seen.add(i)
    assert seen == set(range(len(nets)))
