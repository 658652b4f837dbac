"""Benchmark of the B200 analytic-element DFN solve.

One step = one complete plain solve (discharge-system assembly, sparse LU,
and the damped Jacobi iteration to convergence at MAX_ERROR = 1e-8) of the
~2,000-fracture network: power-law radii (alpha 2.6, 0.5-20 m), Fisher
(kappa 5) normals, log10 T ~ N(-5, 1), heads 1 / 0 on the x faces, ncoef 20,
nint 40, discharge_int 50.  The literal 2,000 discs in a 100 m cube do not
percolate, so 5,500 discs are drawn in a 50 m cube (seed 5) and the largest
cluster joining both heads is kept (2,118 fractures, 5,376 elements; it
converges in 90 outer iterations -- like the reference, some seeds of this
recipe do not converge, so the seed is fixed).

value: solves/s with the network resident in HBM (handle API), timed with
CUDA events on the library's stream, L2 flushed (256 MiB write) between steps.
e2e:   solves/s through the one-call C ABI (andfn_b200_solve) from host
records, host<->device copies included.
--impl reference: the CPU oracle (a C + OpenMP restatement of the reference's
Numba solver with SciPy's SuperLU) on all host cores, each step one complete
solve of the same network (about 8 s on 16 cores).

Multi-GPU (torchrun): every rank solves its own copy of the network
(independent replicas; the solve has no exchange step).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "batched vs plain DFN solves/s at 1e-8 BC residual; adjoint/forward time ratio"
WORKLOAD = ("plain solve: 2,118-fracture spanning cluster of 5,500 power-law/Fisher discs in a 50 m cube "
            "(seed 5), ncoef 20, nint 40, discharge_int 50, MAX_ERROR 1e-8")
MAX_ERROR = 1e-8


def build_network(seed=5):
    from andfn_b200 import network as nw
    net = nw.power_law_fisher(seed, nf=5500, L=50.0, ncoef=20, nint=40)
    return nw.to_records(net)


def constants():
    from andfn_b200.records import default_constants
    return default_constants(MAX_ITERATIONS=200, MAX_ERROR=MAX_ERROR, MAX_NCOEF=20)


BATCH_R = 256
BATCH_WORKLOAD = ("batched: 256 realizations, each N_gen ~ U{200..800} power-law/Fisher discs in a 40 m cube "
                  "(seeds 1000..1255), heads 1 / 0 on the x faces, the clusters touching a head face kept, 4 wells "
                  "(r 0.05 m) with prescribed discharge Q ~ U[-1e-4, 1e-4] m^3/s at random points of random kept "
                  "fractures, ncoef 15, nint 30, discharge_int 50, MAX_ERROR 1e-8")


def build_batch(R=BATCH_R, seed0=1000):
    from andfn_b200 import network as nw
    return nw.to_records_batch([nw.batch_realization(seed0 + i) for i in range(R)])


def batch_constants():
    from andfn_b200.records import default_constants
    return default_constants(MAX_ITERATIONS=200, MAX_ERROR=MAX_ERROR, MAX_NCOEF=15)


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def algorithmic_work(F, E, D):
    """Per-launch algorithmic FP64 flops of the evaluation kernels and bytes
    of the triangular solve (pair cost P(e') = 8(m'-1) + 2 + M + R + L + 2 with
    M = 48 (line) / 4 (circle), R = 11 (Laurent), L = 20 (discharge types))."""
    ty, m, n = E["_type"], E["ncoef"], E["nint"]
    P = np.zeros(len(E))
    line = np.isin(ty, (0, 3, 5))
    P += np.where(m > 0, 8.0 * (m - 1) + 2, 0.0)
    P += np.where(line, 48.0, 4.0)
    P += np.where(np.isin(ty, (0, 3, 4, 5)), 11.0, 0.0)
    P += np.where(np.isin(ty, (0, 2, 3)), 20.0, 0.0)
    P += 2.0
    psum = np.zeros(len(F))
    for f in range(len(F)):
        els = F["elements"][f, : F["nelements"][f]]
        psum[f] = P[els].sum()
    sweep = rhs = dft = 0.0
    for e in range(len(E)):
        if ty[e] == 2:
            continue
        sides = [E["frac0"][e]] + ([E["frac1"][e]] if ty[e] == 0 else [])
        for f in sides:
            sweep += n[e] * (psum[f] - P[e])
            dft += 4.0 * n[e] * m[e]
            if ty[e] in (0, 3):
                rhs += D * psum[f]
    for e in np.nonzero(ty == 2)[0]:
        rhs += D * psum[E["frac0"][e]]
    # head vector from power sums: per (row side, source) pair, ncoef entries of
    # S (16 B) and their coefficient index (4 B) plus the gathered coefficient
    # (16 B); see head_vector_kernel
    entries = 0
    de = np.nonzero(np.isin(ty, (0, 2, 3)))[0]
    msum = np.zeros(len(F))
    for f in range(len(F)):
        els = F["elements"][f, : F["nelements"][f]]
        msum[f] = m[els][ty[els] != 2].sum()
    for e in de:
        entries += msum[E["frac0"][e]] + (msum[E["frac1"][e]] if ty[e] == 0 else 0)
    return {"eval_sweep_flops": sweep, "eval_rhs_flops": rhs, "update_flops": dft,
            "head_vector_bytes": 36.0 * entries, "head_vector_entries": int(entries)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except Exception:
        return {}


def cpu_solve(F, E, D, c, threads=None):
    """One complete solve of the network by the oracle (assembly, SuperLU
    factorisation, iterations to convergence) on the host cores; wall time."""
    from oracle import oracle as orc
    if threads:
        orc.set_num_threads(threads)
    Fs, Es = F.copy(), E.copy()
    st = {}
    t0 = time.perf_counter()
    orc.solve(Fs, Es, D, c, stats=st)
    wall = time.perf_counter() - t0
    return {"seconds_per_solve": wall, "threads": st["threads"], "iterations": int(st["iterations"]),
            "status": int(st.get("status", 0))}


def run_reference(args):
    """The reference arm: the CPU oracle (a C + OpenMP restatement of the
    reference's Numba solve, with SciPy's SuperLU) solving the plain-solve
    network completely in every step, on all host cores."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    F, E = build_network()
    c = constants()
    D = 50
    for _ in range(args.warmup):
        cpu_solve(F, E, D, c)
    secs = []
    r = {}
    for _ in range(args.steps):
        r = cpu_solve(F, E, D, c)
        secs.append(r["seconds_per_solve"])
    v = args.steps / float(np.sum(secs))
    sample = (f"oracle (C+OpenMP restatement of the reference's Numba solve, SciPy SuperLU): one complete solve "
              f"per step (assembly, LU, {r['iterations']} outer iterations to MAX_ERROR 1e-8)")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / v, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": {"workload": WORKLOAD, "parallelism": "cpu threads"},
            "cpu_baseline": {"value": v, "unit": "solves/s", "cores": r["threads"], "kind": "port",
                             "sample": sample},
            "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "step_s": [round(x, 3) for x in secs]}
    print(json.dumps(line), flush=True)


def run_gpu(args):
    import torch
    ws, rank, local = dist_env()
    if ws > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    device = local if ws > 1 else 0
    torch.cuda.set_device(device)
    import andfn_b200
    from andfn_b200 import _ffi
    F, E = build_network()
    c = constants()
    D = 50
    # FP64 roofline denominator
    fp64 = ctypes_double()
    _ffi.check(_ffi.lib().andfn_b200_fp64_peak(device, ctypes_ref(fp64)))
    fp64_tflops = fp64.value
    solver = andfn_b200.Solver(F, E, D, device=device)
    stream = torch.cuda.ExternalStream(solver.stream())
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{device}")
    for _ in range(args.warmup):
        solver.reset()
        solver.run(c)
    torch.cuda.synchronize()
    if args.track_only:
        # streamline tracking alone on the solved network (a profiling case)
        if rank == 0:
            print(json.dumps({"tracking": run_tracking(solver, F, E, reps=1, cpu_particles=0,
                                                       n=args.track_particles, max_length=args.track_max_length)}),
                  flush=True)
        solver.close()
        return
    clocks = ClockSampler(device)
    clocks.start()
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    step_ms = []
    launches = 0
    stats = {}
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        solver.reset()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        stats = solver.run(c)
        b.record(stream)
        b.synchronize()
        step_ms.append(a.elapsed_time(b))
        launches += stats["gpu_launches"]
    torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    clk = clocks.stop()
    # per-kernel times from two more (untimed) solves with event profiling:
    # the events are extra graph nodes, so the timed steps run without them
    solver.set_profiling(True)
    for _ in range(2):
        solver.reset()
        solver.run(c)
    kt = solver.kernel_times()
    solver.set_profiling(False)
    resid = solver.bc_residual()  # of the last timed solve's converged state
    total_ms = float(np.sum(step_ms))
    total_ms, value = aggregate_ranks(total_ms, args.steps, ws, f"cuda:{device}")
    # e2e: one-call C ABI from host records
    e2e_ms = []
    e2e_phases = []
    h2d = d2h = 0
    n_e2e = max(3, min(args.steps, 5))
    for i in range(1 + n_e2e):  # the first call is an untimed warm-up
        Fh, Eh = F.copy(), E.copy()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        andfn_b200.solve(Fh, Eh, D, c)
        dt = (time.perf_counter() - t0) * 1e3
        if i == 0:
            continue
        e2e_ms.append(dt)
        ls = andfn_b200.last_stats
        e2e_phases.append({k: round(ls[k], 2) for k in ("ms_upload", "ms_create_upload", "ms_create_tables",
                                                       "ms_create_order", "ms_setup", "ms_factor", "ms_iterate",
                                                       "ms_download", "ms_alloc", "ms_total")})
        h2d = ls["h2d_bytes"]
        d2h = ls["d2h_bytes"]
    # median: host-side phases share the box's CPUs with other jobs, so a
    # single call can be delayed by seconds; every sample is reported
    e2e_val = ws * 1e3 / float(np.median(e2e_ms))
    # roofline of the dominant kernel
    work = algorithmic_work(F, E, D)
    peaks = measured_peaks()
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    dom = max(kt, key=lambda k: kt[k][0])
    per = {k: (v[0] / v[1] if v[1] else None) for k, v in kt.items()}
    nnz = stats.get("nnz_factors", 0)
    N = stats.get("n_unknowns", 0)
    # factor bytes read per solve: sparse entries (int32 column + f64 value),
    # the dense tail's K^2 used entries (strict lower of L + upper of U) and
    # per-row tables; nnz_factors counts the tail as 2 K^2 and the diagonal once
    K = int(stats.get("dense_tail", 0))
    inverse = int(stats.get("explicit_inverse", 0)) == 1
    if inverse:
        # two passes over the explicit inverse (rows padded to a multiple of 32),
        # A's entries for the residual (value + column, 12 B) and the vectors
        # one pass over the explicit inverse (rows padded to a multiple of 32)
        # per solve, plus the residual (A's entries: value + column, 12 B) and a
        # second pass for the solves that took the refinement step
        ldw = (N + 31) // 32 * 32
        frac_ref = stats.get("refined_solves", 0) / max(1, stats.get("iterations", 1))
        # the refinement pass reads the float copy of the inverse when there is one
        ref_entry = 4.0 if int(stats.get("refine_f32", 0)) == 1 else 8.0
        tri_bytes = (8.0 * N * ldw + frac_ref * ref_entry * N * ldw + (1.0 + frac_ref) * 4.0 * 8 * N
                     + frac_ref * 12.0 * stats.get("nnz_matrix", 0))
        tri_note = (f"explicit inverse: one streaming pass per solve (f64), a residual SpMV and a second pass "
                    f"({'f32' if ref_entry == 4.0 else 'f64'} copy) in {100 * frac_ref:.0f}% of the solves "
                    f"(the refinement step)")
    else:
        tri_bytes = 12.0 * (nnz - 2.0 * K * K - N) + 8.0 * K * K + 24.0 * N
        tri_note = "latency-bound dependency chain (levels of L and U)"
    roof = {}
    # DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one launch
    # on this workload, from ncu captures of the plain-solve profile case
    # (discharge solve: the double pass, plus the refinement pass over the
    # float copy, or a second double pass without one, in the solves that
    # refine); mean of two launches each of the capture
    # `ncu --metrics gpu__time_duration.sum,dram__bytes_read.sum,dram__bytes_write.sum
    #  -k regex:winv_gemv -s 8 -c 4 python bench.py --profile-case plain --profile-iterations 30`
    pass64 = 231325056.0 + 2604416.0
    pass32 = 115852928.0 + 663040.0
    ref_pass = pass32 if inverse and int(stats.get("refine_f32", 0)) == 1 else pass64
    measured_traffic = {"eval_sweep": 111.6e6 + 3.6e6,
                        "trisolve": pass64 + frac_ref * ref_pass if inverse else None}
    if dom in ("eval_sweep", "eval_rhs"):
        fl = work["eval_sweep_flops"] if dom == "eval_sweep" else work["eval_rhs_flops"]
        ach = fl / (per[dom] * 1e-3) / 1e12
        roof = {"kernel": dom, "bound": "fp64", "achieved": ach, "peak": fp64_tflops, "unit": "TFLOP/s",
                "frac": ach / fp64_tflops,
                "traffic": measured_traffic.get(dom) if F is not None and len(F) == 2118 else None,
                "traffic_unit": "B per launch (ncu dram read + write)",
                "peak_source": "measured FP64 FMA probe"}
    else:
        bytes_ = tri_bytes if dom == "trisolve" else 0.0
        ach = bytes_ / (per[dom] * 1e-3) / 1e9
        roof = {"kernel": dom, "bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                "traffic": measured_traffic.get(dom) if len(F) == 2118 else None,
                "traffic_unit": "B per launch (ncu dram read + write)",
                "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)",
                "note": tri_note if dom == "trisolve" else ""}
    ev = {}
    if per.get("eval_sweep"):
        fl = work["eval_sweep_flops"]
        ev["eval_sweep"] = {"achieved_tflops": fl / (per["eval_sweep"] * 1e-3) / 1e12,
                            "frac_of_fp64": fl / (per["eval_sweep"] * 1e-3) / 1e12 / fp64_tflops,
                            "avg_us": per["eval_sweep"] * 1e3}
    if per.get("eval_rhs"):
        gbs = work["head_vector_bytes"] / (per["eval_rhs"] * 1e-3) / 1e9
        ev["head_vector"] = {"achieved_gbs": gbs, "frac_of_hbm": gbs / hbm, "bytes": work["head_vector_bytes"],
                             "avg_us": per["eval_rhs"] * 1e3,
                             "note": "power-sum gather; the sums (36 B per entry) stay L2-resident"}
    ev["discharge_solve"] = {"mode": "explicit inverse" if inverse else "triangular solves", "bytes": tri_bytes,
                             "dense_tail": K, "note": tri_note}
    if per.get("trisolve"):
        gbs = tri_bytes / (per["trisolve"] * 1e-3) / 1e9
        ev["discharge_solve"].update({"avg_us": per["trisolve"] * 1e3, "achieved_gbs": gbs, "frac_of_hbm": gbs / hbm})
    tracking = None
    if not args.no_track and rank == 0:
        try:
            tracking = run_tracking(solver, F, E)
        except Exception as exc:  # reported in the line; the solve numbers stand without it
            tracking = {"error": f"{type(exc).__name__}: {exc}"}
    batched = None if args.no_batch else run_batched(args, device, flush)
    adjoint = None if args.no_adjoint else run_adjoint(args, device, F, E)
    large = None if args.no_large else run_large(args, device)
    if rank == 0:
        cpu = None
        if not args.no_cpu:
            r = cpu_solve(F, E, D, c)
            cpu = {"value": 1.0 / r["seconds_per_solve"], "unit": "solves/s", "cores": r["threads"], "kind": "port",
                   "sample": f"oracle: one complete solve ({r['seconds_per_solve']:.1f} s, {r['iterations']} "
                             f"iterations, status {r['status']})"}
        line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
                "step_ms": [round(x, 3) for x in step_ms], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
                "config": {"workload": WORKLOAD, "fractures": int(len(F)), "elements": int(len(E)),
                           "iterations": int(stats["iterations"]), "n_unknowns": int(N), "nnz_lu": int(nnz),
                           "l2": "flushed (256 MiB write) between steps", "parallelism": f"replicas x{ws}"},
                "e2e": {"value": e2e_val, "unit": "solves/s", "h2d_bytes_per_step": int(h2d),
                        "d2h_bytes_per_step": int(d2h), "statistic": "median", "ms": [round(x, 2) for x in e2e_ms],
                        "phases_ms": e2e_phases},
                "gpu_launches": int(launches), "roofline": roof, "kernels_us": {k: (v * 1e3 if v else None) for k, v in per.items()},
                "kernel_share": {k: kt[k][0] / max(1e-12, sum(v[0] for v in kt.values())) for k in kt},
                "eval_roofline": ev, "phase_ms": {k: stats[k] for k in ("ms_setup", "ms_factor", "ms_factor_sparse",
                                                                 "ms_factor_dense", "ms_factor_levels",
                                                                 "ms_inverse", "ms_iterate")},
                "fp64_peak_tflops": fp64_tflops, "clocks": clk, "cpu_baseline": cpu, "batched": batched,
                "bc_residual": {"max": resid["bc_max"], "worst_element": int(resid["bc_worst"]),
                                "element_type": int(E["_type"][resid["bc_worst"]]) if resid["bc_worst"] >= 0 else None,
                                "flux_imbalance_max": resid["flux_max"], "h_scale": resid["h_scale"],
                                "q_scale": resid["q_scale"],
                                "note": "series truncation residual at the collocation points (ncoef 20); "
                                        "convergence uses the reference's MAX_ERROR rule"},
                "adjoint": adjoint, "large": large, "tracking": tracking}
        # the headline ratios, last so that a truncated copy of the line keeps them
        line["headline"] = headline_summary(value, e2e_val, cpu, roof, batched, adjoint, large)
        print(json.dumps(line), flush=True)
    solver.close()
    if ws > 1:
        torch.distributed.destroy_process_group()


def headline_summary(value, e2e, cpu, roof, batched, adjoint, large):
    """Plain GPU vs CPU solves/s (device-resident and end to end), batched
    per-realization rate vs the plain single-network rate, gradient time vs
    forward time, the finite-difference check and the dominant kernel's
    roofline fraction."""
    out = {"plain_solves_per_s": value, "e2e_solves_per_s": e2e}
    if cpu:
        out.update({"cpu_solves_per_s": cpu["value"], "value_over_cpu": value / cpu["value"],
                    "e2e_over_cpu": e2e / cpu["value"], "cpu_cores": cpu["cores"]})
    if batched:
        out.update({"batched_realizations_per_s": batched["value"],
                    "batched_speedup_vs_plain": batched["speedup_vs_plain"]})
    if adjoint:
        out["gradient_over_forward"] = adjoint["gradient_over_forward"]
        fd = adjoint.get("fd_check")
        if fd:
            out["fd_max_rel_err"] = {str(x["step"]): x["max_rel_err"] for x in fd["steps"]}
    if large:
        out["large_gradient_over_forward"] = large["gradient_over_forward"]
    if roof:
        out["roofline"] = {"kernel": roof.get("kernel"), "frac": roof.get("frac")}
    return out


def run_batched(args, device, flush, sample=32):
    """Batched realizations: one BatchSolver run over all of them against the
    same realizations solved one at a time by the plain handle API (a sample
    of them, timed the same way).  Under torchrun the realizations are split
    across the ranks (longest processing time first by sweep pairs,
    andfn_b200.shard); each rank solves its share, the value uses the slowest
    rank's time."""
    import torch
    import andfn_b200
    from andfn_b200.shard import partition_lpt, sweep_pairs
    ws, rank, _ = dist_env()
    recs_all = build_batch()
    parts = partition_lpt([sweep_pairs(F, E) for F, E in recs_all], ws)
    recs = [recs_all[i] for i in parts[rank]]
    c = batch_constants()
    D = 50
    bs = andfn_b200.BatchSolver([(F.copy(), E.copy()) for F, E in recs], D, device=device)
    stream = torch.cuda.ExternalStream(bs.stream())
    for _ in range(args.warmup):
        bs.run(c)
    torch.cuda.synchronize()
    ms = []
    st = []
    launches = 0
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        st = bs.run(c)
        b.record(stream)
        b.synchronize()
        ms.append(a.elapsed_time(b))
        launches += st[0]["gpu_launches"]
    bs.set_profiling(True)  # per-kernel times from two more untimed runs
    for _ in range(2):
        bs.run(c)
    kt = bs.kernel_times()
    bs.close()
    R = len(recs_all)
    total_ms, _ = aggregate_ranks(float(np.sum(ms)), args.steps, ws, f"cuda:{device}")
    value = R * args.steps / (total_ms / 1e3)
    # the same realizations through the plain single-network path
    plain_ms = []
    for F, E in recs[:sample]:
        with andfn_b200.Solver(F.copy(), E.copy(), D, device=device) as s1:
            s1.run(c)  # warm-up
            flush.zero_()
            torch.cuda.synchronize()
            st1 = torch.cuda.ExternalStream(s1.stream())
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(st1)
            s1.run(c)
            b.record(st1)
            b.synchronize()
            plain_ms.append(a.elapsed_time(b))
    plain_rate = len(plain_ms) / (float(np.sum(plain_ms)) / 1e3)
    # end to end from host records (one call per batch)
    e2e = []
    for i in range(4):  # the first call is an untimed warm-up
        nets = [(F.copy(), E.copy()) for F, E in recs]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sts = andfn_b200.solve_batch(nets, D, c)
        if i:
            e2e.append(time.perf_counter() - t0)
    e2e_s, _ = aggregate_ranks(float(np.median(e2e)) * 1e3, 1, ws, f"cuda:{device}")
    its = np.array([x["iterations"] for x in st])
    status = np.array([x["status"] for x in st])
    return {"workload": BATCH_WORKLOAD, "realizations": R, "realizations_this_rank": len(recs),
            "fractures": int(sum(len(F) for F, _ in recs_all)), "elements": int(sum(len(E) for _, E in recs_all)),
            "value": value, "unit": "realizations/s", "ms_per_step": total_ms / args.steps,
            "step_ms": [round(x, 3) for x in ms],
            "gpu_launches_per_step": launches / args.steps,
            "sharding": f"{ws} rank(s), longest processing time first by sweep pairs",
            "e2e": {"value": R / (e2e_s / 1e3), "unit": "realizations/s", "statistic": "median, slowest rank",
                    "ms": [round(1e3 * x, 2) for x in e2e],
                    "h2d_bytes_per_step": int(sts[0]["h2d_bytes"]), "d2h_bytes_per_step": int(sts[0]["d2h_bytes"])},
            "plain_sequential": {"value": plain_rate, "unit": "realizations/s", "sample": len(plain_ms),
                                 "ms_per_realization": float(np.mean(plain_ms))},
            "speedup_vs_plain": value / ws / plain_rate,
            "iterations": {"max": int(its.max()), "mean": float(its.mean())},
            "status_counts": {str(k): int(v) for k, v in zip(*np.unique(status, return_counts=True))},
            "phase_ms": {k: st[0][k] for k in ("ms_setup", "ms_factor", "ms_iterate")},
            "kernels_ms_per_run": {k: v[0] / 2 for k, v in kt.items()},
            "kernels_note": "per-kernel device time of one batched run (two untimed runs with event profiling)"}


ADJ_WORKLOAD = ("adjoint: the plain-solve network + 50 observation points (uniform on random fractures, seed 7), "
                "h_obs = forward heads + N(0, 0.01); J = sum (h - h_obs)^2 + discharge through the x = L face; "
                "dJ/dlog t of every fracture through torch.autograd")


def run_adjoint(args, device, F, E, fd_fracs=20, fd_its=400, steps_fd=(1e-6, 1e-4)):
    """Gradient of the head-misfit + outflow objective w.r.t. log t of all
    fractures: time of the backward pass against the forward solve, and a
    central finite-difference check on fd_fracs random fractures among those
    whose gradient is at least 1e-3 of the largest (smaller entries are below
    the round-off of J in a difference quotient) (forward solves of a fixed
    fd_its iterations for the check, so J is a smooth function of log t), at
    each step in steps_fd."""
    import torch
    from andfn_b200.adjoint import DFNModel
    from andfn_b200.records import default_constants
    D = 50
    dev = f"cuda:{device}"
    rng = np.random.default_rng(7)
    n_obs = 50
    fr = rng.integers(0, len(F), n_obs)
    z = F["radius"][fr] * 0.9 * np.sqrt(rng.uniform(size=n_obs)) * np.exp(2j * np.pi * rng.uniform(size=n_obs))
    frt = torch.tensor(fr, dtype=torch.int64, device=dev)
    zt = torch.tensor(z, dtype=torch.complex128, device=dev)
    outlet = torch.tensor(np.nonzero((E["_type"] == 3) & (E["head"] == 0.0))[0], device=dev)
    logt0 = np.log(F["t"].astype(np.float64))

    def objective(model, hobs, lt):
        coef, q, C = model.solve(lt)
        h = model.heads(coef, q, C, lt, frt, zt)
        return ((h - hobs) ** 2).sum() + q[outlet].sum(), h

    out = {"workload": ADJ_WORKLOAD, "observations": n_obs}
    model = DFNModel(F.copy(), E.copy(), constants(), D, device=device, adjoint_tol=1e-8)
    lt = torch.tensor(logt0, dtype=torch.float64, device=dev)
    with torch.no_grad():
        _, h0 = objective(model, torch.zeros(n_obs, dtype=torch.float64, device=dev), lt)
    hobs = h0 + torch.tensor(rng.normal(0.0, 0.01, n_obs), device=dev)
    fwd, bwd, its, adj_its = [], [], [], []
    for i in range(args.warmup + args.steps):
        ltg = lt.clone().requires_grad_(True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        J, _ = objective(model, hobs, ltg)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        J.backward()
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        if i >= args.warmup:
            fwd.append(t1 - t0)
            bwd.append(t2 - t1)
            its.append(model.stats["iterations"])
            adj_its.append(model.adjoint_stats["iterations"])
    g = ltg.grad.detach().cpu().numpy()
    # medians: the forward's factorisation runs on host cores shared with other jobs
    out.update({"forward_ms": 1e3 * float(np.median(fwd)), "gradient_ms": 1e3 * float(np.median(bwd)),
                "gradient_over_forward": float(np.median(bwd) / np.median(fwd)), "statistic": "median",
                "forward_samples_ms": [round(1e3 * x, 2) for x in fwd],
                "gradient_samples_ms": [round(1e3 * x, 2) for x in bwd],
                "forward_iterations": int(its[-1]), "adjoint_iterations": int(adj_its[-1]),
                "adjoint_tol": 1e-8, "adjoint_status": int(model.adjoint_stats["status"]),
                "grad_norm": float(np.linalg.norm(g))})
    model.close()
    if fd_fracs > 0:
        cfd = default_constants(MAX_ITERATIONS=fd_its, MAX_ERROR=1e-300, MAX_NCOEF=20)
        m2 = DFNModel(F.copy(), E.copy(), cfd, D, device=device, adjoint_tol=1e-10)
        ltg = lt.clone().requires_grad_(True)
        J, _ = objective(m2, hobs, ltg)
        J.backward()
        ga = ltg.grad.detach().cpu().numpy()
        cand = np.nonzero(np.abs(ga) >= 1e-3 * np.abs(ga).max())[0]
        sel = np.random.default_rng(20).choice(cand, size=min(fd_fracs, len(cand)), replace=False)
        checks = []
        with torch.no_grad():
            for h_fd in steps_fd:
                gf = np.zeros(len(sel))
                for k, f in enumerate(sel):
                    vals = []
                    for sgn in (1.0, -1.0):
                        l2 = logt0.copy()
                        l2[f] += sgn * h_fd
                        Jv, _ = objective(m2, hobs, torch.tensor(l2, dtype=torch.float64, device=dev))
                        vals.append(float(Jv))
                    gf[k] = (vals[0] - vals[1]) / (2 * h_fd)
                rel = np.abs(ga[sel] - gf) / np.abs(gf)
                checks.append({"step": h_fd, "max_rel_err": float(rel.max()), "median_rel_err": float(np.median(rel)),
                               "max_err_over_max_grad": float(np.abs(ga[sel] - gf).max() / np.abs(ga).max())})
        out["fd_check"] = {"fractures": int(len(sel)), "candidates": int(len(cand)),
                           "selection": "random (seed 20) among |dJ/dlog t| >= 1e-3 max",
                           "forward_iterations": fd_its, "adjoint_iterations": int(m2.adjoint_stats["iterations"]),
                           "adjoint_status": int(m2.adjoint_stats["status"]), "steps": checks}
        m2.close()
    return out


LARGE_WORKLOAD = ("large: 20,000 power-law/Fisher discs (radii 1-40 m) in a 200 m cube (seed 11), largest cluster "
                  "joining both head planes (2,588 fractures), 100 impermeable circles (radius 1-3 m), bounding "
                  "circles on every fracture, ncoef 30, nint 60, MAX_ERROR 1e-8; forward solve + gradient of 50 "
                  "observation heads + outflow w.r.t. log t")


def run_large(args, device):
    """Forward solve and log-transmissivity gradient of the large network."""
    import torch
    from andfn_b200 import network as nw
    from andfn_b200.adjoint import DFNModel
    from andfn_b200.records import default_constants
    F, E = nw.to_records(nw.large_network())
    c = default_constants(MAX_ITERATIONS=300, MAX_ERROR=MAX_ERROR, MAX_NCOEF=30)
    dev = f"cuda:{device}"
    rng = np.random.default_rng(17)
    fr = rng.integers(0, len(F), 50)
    z = F["radius"][fr] * 0.8 * np.sqrt(rng.uniform(size=50)) * np.exp(2j * np.pi * rng.uniform(size=50))
    frt = torch.tensor(fr, dtype=torch.int64, device=dev)
    zt = torch.tensor(z, dtype=torch.complex128, device=dev)
    outlet = torch.tensor(np.nonzero((E["_type"] == 3) & (E["head"] == 0.0))[0], device=dev)
    free0, total = torch.cuda.mem_get_info(device)
    model = DFNModel(F.copy(), E.copy(), c, 50, device=device, adjoint_tol=1e-8)
    lt0 = torch.tensor(np.log(F["t"]), dtype=torch.float64, device=dev)
    with torch.no_grad():
        coef, q, C = model.solve(lt0)
        hobs = model.heads(coef, q, C, lt0, frt, zt) + torch.tensor(rng.normal(0, 0.01, 50), device=dev)
    fwd, bwd = [], []
    for i in range(1 + max(1, min(args.steps, 2))):
        lt = lt0.clone().requires_grad_(True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        coef, q, C = model.solve(lt)
        h = model.heads(coef, q, C, lt, frt, zt)
        J = ((h - hobs) ** 2).sum() + q[outlet].sum()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        J.backward()
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        if i:
            fwd.append(t1 - t0)
            bwd.append(t2 - t1)
    free1, _ = torch.cuda.mem_get_info(device)
    st, ast = model.stats, model.adjoint_stats
    model.close()
    return {"workload": LARGE_WORKLOAD, "fractures": int(len(F)), "elements": int(len(E)),
            "n_unknowns": int(st["n_unknowns"]), "dense_tail": int(st["dense_tail"]),
            "forward_iterations": int(st["iterations"]), "forward_status": int(st["status"]),
            "forward_ms": 1e3 * float(np.median(fwd)), "gradient_ms": 1e3 * float(np.median(bwd)),
            "gradient_over_forward": float(np.median(bwd) / np.median(fwd)), "statistic": "median",
            "adjoint_sweeps": int(ast["iterations"]), "adjoint_residual": float(ast["residual"]),
            "adjoint_status": int(ast["status"]), "device_memory_mb": (free0 - free1) / 2**20,
            "grad_norm": float(torch.linalg.norm(lt.grad).item())}


TRACK_PARTICLES, TRACK_MAX_LENGTH, TRACK_DS = 8192, 1000, 1e-2


def run_tracking(solver, F, E, reps=3, cpu_particles=2, seed=9, n=TRACK_PARTICLES, max_length=TRACK_MAX_LENGTH):
    """Streamline tracking on the solved plain-solve network: TRACK_PARTICLES
    particles (seeded starts at r <= 0.9 R on random fractures, elevations
    U(0, 1), apertures 10^U(-4, -3)) traced forward, up to TRACK_MAX_LENGTH
    points each, by one andfn_b200_track launch.  Timed end to end through the
    public call (host buffers, copies and allocation inside; the call returns
    after its stream has synchronised), median of reps.  CPU leg: the oracle's
    tracker (a pure-Python port of the reference's pure-Python tracking) on the
    first cpu_particles particles."""
    from andfn_b200.track import track
    from oracle import track as ot
    rng = np.random.default_rng(seed)
    ap = 10 ** rng.uniform(-4, -3, len(F))
    fr = rng.integers(0, len(F), n)
    z = np.sqrt(rng.uniform(0, 0.81, n)) * F["radius"][fr] * np.exp(1j * rng.uniform(0, 2 * np.pi, n))
    el = rng.uniform(0, 1, n)
    track(solver, ap, fr[:64], z[:64], el[:64], TRACK_DS, max_length)
    ms = []
    for _ in range(reps):
        t0 = time.perf_counter()
        tr = track(solver, ap, fr, z, el, TRACK_DS, max_length)
        ms.append((time.perf_counter() - t0) * 1e3)
    med = float(np.median(ms))
    pts = int(tr.npoints.sum())
    Fs, Es = F.copy(), E.copy()
    solver.download(Fs, Es)
    t0 = time.perf_counter()
    cpu_pts = 0
    for i in range(cpu_particles):
        seg, _, _, _ = ot.streamline_tracking(Fs, Es, ap, z[i], int(fr[i]), float(el[i]), TRACK_DS, max_length)
        cpu_pts += sum(len(x) for x in seg)
    cpu_s = max(time.perf_counter() - t0, 1e-9)
    return {"particles": n, "max_length": max_length, "ds": TRACK_DS, "points": pts,
            "ms": [round(x, 2) for x in ms], "particles_per_s": n / (med * 1e-3), "points_per_s": pts / (med * 1e-3),
            "statistic": "median, end to end through andfn_b200_track (host buffers)",
            "truncated": int((tr.status != 0).sum()), "ended_on_element": int((tr.element >= 0).sum()),
            "cpu_baseline": {"points_per_s": cpu_pts / cpu_s, "particles": cpu_particles, "points": cpu_pts,
                             "cores": 1, "kind": "port", "sample": "oracle/track.py on the first particles"}}


def run_profile_case(args):
    """One untimed run of a bench workload, the command profiler captures
    wrap: ``plain`` (one solve of the plain-solve network through the one-call
    C ABI), ``adjoint`` (one forward solve plus the gradient of the head-misfit
    + outflow objective w.r.t. log t) or ``batch`` (one batched solve of the
    256 realizations).  --profile-iterations caps MAX_ITERATIONS.  The
    iterations run as 8-iteration graph launches from the host (not the
    single device-side loop), whose kernels a profiler attributes one by one."""
    os.environ.setdefault("ANDFN_B200_DEVICE_LOOP", "0")
    import andfn_b200
    its = args.profile_iterations
    if args.profile_case == "batch":
        recs = build_batch()
        c = batch_constants()
        if its:
            c["MAX_ITERATIONS"] = its
        st = andfn_b200.solve_batch(recs, 50, c)
        it = [s["iterations"] for s in st]
        print(f"realizations {len(st)} iterations max {max(it)} mean {np.mean(it):.1f}", flush=True)
        return
    F, E = build_network()
    c = constants()
    if its:
        c["MAX_ITERATIONS"] = its
    if args.profile_case == "adjoint":
        import torch
        from andfn_b200.adjoint import DFNModel
        rng = np.random.default_rng(7)
        fr = rng.integers(0, len(F), 50)
        z = F["radius"][fr] * 0.9 * np.sqrt(rng.uniform(size=50)) * np.exp(2j * np.pi * rng.uniform(size=50))
        dev = "cuda:0"
        frt = torch.tensor(fr, device=dev)
        zt = torch.tensor(z, dtype=torch.complex128, device=dev)
        outlet = torch.tensor(np.nonzero((E["_type"] == 3) & (E["head"] == 0.0))[0], device=dev)
        m = DFNModel(F.copy(), E.copy(), c, 50, adjoint_tol=1e-8)
        lt = torch.tensor(np.log(F["t"]), device=dev, requires_grad=True)
        coef, q, C = m.solve(lt)
        h = m.heads(coef, q, C, lt, frt, zt)
        J = ((h - 0.5) ** 2).sum() + q[outlet].sum()
        J.backward()
        print(f"forward iterations {m.stats['iterations']} adjoint sweeps {m.adjoint_stats['iterations']} "
              f"residual {m.adjoint_stats['residual']:.2e}", flush=True)
        m.close()
        return
    andfn_b200.solve(F, E, 50, c)
    st = andfn_b200.last_stats
    print(f"iterations {st['iterations']} status {st['status']} factor {st['ms_factor']:.1f} ms "
          f"iterate {st['ms_iterate']:.1f} ms", flush=True)


def aggregate_ranks(total_ms: float, steps: int, world_size: int, device=None) -> tuple[float, float]:
    """Slowest rank's timed milliseconds (all-reduce MAX) and the whole-job
    value: every rank solves its own network, so value = world_size * steps
    / max time."""
    if world_size > 1:
        import torch
        import torch.distributed as dist
        t = torch.tensor([total_ms], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    return total_ms, world_size * steps / (total_ms / 1e3)


def ctypes_double():
    import ctypes
    return ctypes.c_double()


def ctypes_ref(x):
    import ctypes
    return ctypes.byref(x)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-realizations measurement")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint (gradient) measurement")
    ap.add_argument("--no-large", action="store_true", help="skip the large-network forward + gradient run")
    ap.add_argument("--no-track", action="store_true", help="skip the streamline-tracking measurement")
    ap.add_argument("--track-only", action="store_true", help="only solve once and time streamline tracking")
    ap.add_argument("--track-particles", type=int, default=TRACK_PARTICLES)
    ap.add_argument("--track-max-length", type=int, default=TRACK_MAX_LENGTH)
    ap.add_argument("--profile-case", choices=["plain", "adjoint", "batch"], default=None,
                    help="one untimed run of that workload (the command a profiler capture wraps); no JSON line")
    ap.add_argument("--profile-iterations", type=int, default=None, help="MAX_ITERATIONS of --profile-case")
    args = ap.parse_args()
    if args.profile_case:
        run_profile_case(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
