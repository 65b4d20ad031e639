#!/usr/bin/env python
"""Searchlight solves/sec on the hemisphere template workload with singular searchlights.

One step = one searchlight Procrustes pass (with scaling) over a hemisphere:
10242 Fibonacci-sphere vertices, nt = 400, one searchlight of 100-300 vertices
per vertex, subject 1 aligned onto subject 0 of the template workload, with
vertex columns duplicated until ~10% of the searchlights are exactly singular;
output the weighted transforms combined into the symmetric CSC/CSR matrix.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

value     the tensor-core solver (split-BF16 products, Newton-Schulz polar) on device-resident
          inputs (float64 X, Y already in HBM), CUDA events around each step on the launching
          stream, L2 flushed (256 MiB write) between steps
plain_fp32  the same step and inputs in the plain FP32 form (FP32 Jacobi, no refinement, no FP64):
          the metric's denominator; mixed_form, fp64_form the other solvers
config2_template_pair  the same pair without duplicated columns (tensor-core and plain FP32)
e2e       the C ABI dense entry point (ha_searchlight_procrustes_dense, backend 4) from
          host float64 buffers into a host nv x nv float64 matrix, wall clock per call; a
          cold first call after ha_b200_cleanup beside it
roofline  dominant kernel (per-kind CUDA event times recorded by the library)
cpu_baseline  the reference C library (oracle/_ref, cpu64 arm, all host threads) on a
          bounded sample of the same searchlights
config4_ridge_grid_full  the ridge grid search over all 40962 searchlights of 50-500 vertices
          (float64, cost grids checked against the oracle on a sample), with its plain FP32
          form on the same inputs as plain_fp32 (winners and costs against float64)
config5_learned  the mixed-precision learned proposal on the held-out subject against the plain
          FP32 full grid on the same searchlights (the float64 grid and learned form beside them)
--no-extras  skips the two config fields (N > 1 runs never have them)
--impl reference  times only the reference CPU implementation (rank 0 of any N)
"""

from __future__ import annotations

import os

# one BLAS thread per OpenMP thread for the reference CPU arm (set before numpy/scipy load BLAS)
os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")

import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "searchlight solves/sec vs plain FP32 GPU form at stated FP64-oracle error"
UNIT = "searchlights/s"
WORKLOAD = "hemisphere_template_pair_10pct_singular"
PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}
FP32_SIMT_NOMINAL_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["b200", "reference"], default="b200")
    p.add_argument("--nv", type=int, default=10242)
    p.add_argument("--nt", type=int, default=400)
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-extras", action="store_true",
                   help="skip the config-4 (full-size grid search) and config-5 (learned proposal) sub-fields")
    p.add_argument("--cpu-seconds", type=float, default=15.0)
    p.add_argument("--workload", choices=["template", "rankdef", "grid", "learned", "shard", "forrest", "refgpu",
                                           "pca"],
                   default="rankdef",
                   help="rankdef (default; 'template' is the same run): the headline Procrustes step on the "
                        "template pair with 10%% singular searchlights, the plain pair as a sub-field; grid: the "
                        "searchlight ridge grid search (40962 vertices, every --grid-step-th searchlight); "
                        "learned: the learned proposal; shard: one "
                        "hemisphere split over the N GPUs (strong scaling); forrest: the shapes of the "
                        "reference's published run (nt 1818, searchlights of 90-170); refgpu: the reference's "
                        "own CUDA arm (oracle/_ref_cuda) against this library on config 1 and the Forrest shape; pca: the "
                        "searchlight PCA template on the template workload's hemisphere (10 subjects)")
    p.add_argument("--grid-step", type=int, default=16)
    p.add_argument("--grid-bits", type=int, choices=[32, 64], default=64,
                   help="grid workload: float64 search (64) or its plain FP32 form (32)")
    p.add_argument("--ref-seconds", type=float, default=0.0,
                   help="reference arm: seconds of CPU work per step (default: 150 s over all steps)")
    return p.parse_args()


def workload(seed, nv, nt):
    from hyperalignment_b200 import workloads as W
    return W.template_procrustes_pair(seed=seed, nv=nv, nt=nt)


def config_dict(w, extra=None):
    sizes = w.sls.sizes
    d = {"workload": WORKLOAD, "nv": w.nv, "nt": w.nt, "searchlights": w.sls.count,
         "sl_size_min": int(sizes.min()), "sl_size_max": int(sizes.max()), "sl_size_mean": round(float(sizes.mean()), 2),
         "scaling": True, "reflection": True, "weights": "linear distance",
         "l2": "flushed between steps (256 MiB write)"}
    if extra:
        d.update(extra)
    return d


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f), "measured"
    return dict(PEAKS_FALLBACK), "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.lines = []
        self.proc = None
        self.th = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, ValueError):
            self.proc = None
            return
        self.th = threading.Thread(target=self._read, daemon=True)
        self.th.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.th:
            self.th.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(smax)), "reasons": sorted(reasons),
                "samples": len(sm)}


def max_over_ranks(value, ws, device=None):
    """The largest per-rank value over all ranks (the job's time); the value itself on one rank."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    if ws > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(ws, units_per_rank, steps, seconds):
    """Whole-job rate of N replicas, each processing units_per_rank per step (weak scaling)."""
    return ws * units_per_rank * steps / seconds


def dist_setup(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# ---------------------------------------------------------------------------------------------
# reference CPU arm
# ---------------------------------------------------------------------------------------------

def reference_rate(w, seconds, threads, start=0, backend=0):
    """Reference dense entry point (backend 0 = cpu64, 1 = cpu32) on a contiguous sample of
    searchlights sized to ~seconds."""
    from oracle import ref_lib as R
    R.set_threads(threads)
    s = w.sls
    # size the sample from a short probe
    probe = s.subset(np.arange(start, min(start + 4 * threads, s.count)))
    Xf, Yf = np.asfortranarray(w.X), np.asfortranarray(w.Y)
    t0 = time.perf_counter()
    _ref_call(R, Xf, Yf, probe, backend)
    dt = time.perf_counter() - t0
    rate = probe.count / max(dt, 1e-6)
    m = int(min(s.count, max(threads, rate * seconds)))
    idx = (start + np.arange(m)) % s.count
    sample = s.subset(idx)
    t0 = time.perf_counter()
    _ref_call(R, Xf, Yf, sample, backend)
    dt = time.perf_counter() - t0
    return sample.count / dt, sample.count, dt


_REF_T = {}


def _ref_call(R, Xf, Yf, sls, backend=0):
    h = R.lib()
    nt, nv = Xf.shape
    T = _REF_T.get(nv)
    if T is None:
        T = _REF_T[nv] = np.zeros((nv, nv))
    rc = h.ha_searchlight_procrustes_dense(
        Xf.ctypes.data_as(R.c_double_p), Yf.ctypes.data_as(R.c_double_p), nt, nv,
        sls.indices.ctypes.data_as(R.c_int32_p), sls.offsets.ctypes.data_as(R.c_int32_p),
        sls.dists.ctypes.data_as(R.c_double_p), sls.count, sls.radius, T.ctypes.data_as(R.c_double_p),
        True, True, backend, True)
    if rc != 0:
        raise RuntimeError(f"reference rc={rc}")


def run_reference(args):
    ws, rank, _ = dist_setup(args)
    if rank != 0:
        return
    from oracle import ref_lib as R
    if not R.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libhyperalignment.so not built"}))
        return
    from hyperalignment_b200 import workloads as W
    w = W.rank_deficient_pair(0, nv=args.nv, nt=args.nt)
    threads = os.cpu_count() or 1
    budget = args.ref_seconds if args.ref_seconds > 0 else max(2.0, 150.0 / max(1, args.steps + args.warmup))
    rates, times, counts = [], [], []
    start = 0
    for i in range(args.warmup + args.steps):
        r, m, dt = reference_rate(w, budget, threads, start)
        start = (start + m) % w.sls.count
        if i >= args.warmup:
            rates.append(r)
            times.append(dt)
            counts.append(m)
    value = float(sum(counts) / sum(times))
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": float(1e3 * np.mean(times)), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_dict(w, {"sample": f"{int(np.mean(counts))} searchlights per step (contiguous, rotating)"}),
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": f"{int(np.mean(counts))} of {w.sls.count} searchlights per step, cpu64 arm, "
                                   f"OpenMP {threads} threads, OPENBLAS_NUM_THREADS=1"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))


# ---------------------------------------------------------------------------------------------
# B200 arm
# ---------------------------------------------------------------------------------------------

def tc_algorithmic_flops(sizes, iters):
    """Tensor-core work of the Newton-Schulz polar iteration as the algorithm defines it (no
    padding): per searchlight and iteration two n x n x n products (X^T X and X P), each executed as
    three FP16 products of the two-part split: 12 n^3 flops."""
    n = sizes.astype(np.float64)
    return float((12.0 * iters.astype(np.float64) * n ** 3).sum())


def tc_executed_flops(sizes, iters):
    """MMA work the iteration's kernels issue, padding included: rows in 128-row tiles, N and K padded
    to 16, three products per n^3 product, two n^3 products per iteration."""
    n = sizes.astype(np.int64)
    npad = (n + 15) // 16 * 16
    mpad = (npad + 127) // 128 * 128
    return float((2 * 3 * 2 * iters.astype(np.float64) * mpad * npad.astype(np.float64) ** 2).sum())


def sample_errors(w, singular, sample, Ts):
    """Per-T and aligned-data (X_sl T) errors vs the float64 oracle; singular searchlights are compared
    on the row space of A (the part of T that A determines) and on X_sl T (unique)."""
    from oracle import ha_oracle as O
    rows = {"singular": [], "regular": []}
    for j, q in enumerate(sample):
        sl = w.sls.indices[w.sls.offsets[q]:w.sls.offsets[q + 1]]
        Xs, Ys = w.X[:, sl], w.Y[:, sl]
        Tref = O.procrustes(Xs, Ys, True, False)
        T = Ts[j]
        XT, XTref = Xs @ T, Xs @ Tref
        if singular is not None and singular[q]:
            A = Xs.T @ Ys
            T, Tref = range_part(T, A), range_part(Tref, A)
        rows["singular" if singular is not None and singular[q] else "regular"].append(
            (np.linalg.norm(T - Tref) / np.linalg.norm(Tref), np.abs(T - Tref).max(),
             np.linalg.norm(XT - XTref) / np.linalg.norm(XTref), np.abs(XT - XTref).max()))
    out = {}
    for k, v in rows.items():
        if not v:
            continue
        e = np.array(v)
        out[k] = {"T_relfrob_max": float(e[:, 0].max()), "T_relfrob_median": float(np.median(e[:, 0])),
                  "T_maxabs_max": float(e[:, 1].max()), "XT_relfrob_max": float(e[:, 2].max()),
                  "XT_maxabs_max": float(e[:, 3].max()), "count": int(e.shape[0])}
    return out


class StepClock:
    """Device timer of the sharded steps: CUDA events on the current stream (GPU ranks) or
    perf_counter (CPU ranks of the gloo tests)."""

    def __init__(self, device):
        import torch
        self.cuda = torch.device(device).type == "cuda"
        self.device = device

    def mark(self):
        import torch
        if self.cuda:
            e = torch.cuda.Event(enable_timing=True)
            e.record(torch.cuda.current_stream(self.device))
            return e
        return time.perf_counter()

    def ms(self, a, b):
        return a.elapsed_time(b) if self.cuda else (b - a) * 1e3

    def sync(self):
        import torch
        if self.cuda:
            torch.cuda.synchronize(self.device)


def sharded_rank(ws, rank, offsets, nv, make_range, steps, warmup, device, flush=None, group=None):
    """The rank code of one hemisphere over ws ranks (strong scaling; hyperalignment_b200/shard.py):
    this rank's contiguous searchlight range (balanced by n^3), its pattern and the column exchange
    are built once; every step zeroes the partial CSC values, solves the range into them and sends
    them to the column owners in one all-to-all.  make_range(lo, hi) -> (indptr, rows, solve) with
    solve(partial) writing the range's weighted local transforms into its CSC pattern.  Times are
    the max over ranks of the per-rank sums over the timed steps."""
    import torch
    import torch.distributed as dist
    from hyperalignment_b200 import shard as S
    b = S.split_searchlights(offsets, ws)
    lo, hi = int(b[rank]), int(b[rank + 1])
    solve = None
    if hi > lo:
        indptr, rows, solve = make_range(lo, hi)
    else:
        indptr, rows = np.zeros(nv + 1, dtype=np.int64), np.zeros(0, dtype=np.int32)
    ex = S.ColumnExchange(indptr, rows, nv, group=group, device=device)
    partial = torch.zeros(int(np.asarray(indptr)[-1]), dtype=torch.float64, device=device)
    clock = StepClock(device)

    def solve_part():
        partial.zero_()
        if solve is not None:
            solve(partial)

    for _ in range(warmup):
        solve_part()
        owned = ex.combine(partial)
    clock.sync()
    if ws > 1:
        dist.barrier(group=group)
    marks = []
    for _ in range(steps):
        if flush is not None:
            flush.zero_()
        a = clock.mark()
        solve_part()
        m = clock.mark()
        owned = ex.combine(partial)
        e = clock.mark()
        marks.append((a, m, e))
    clock.sync()
    job = max_over_ranks(sum(clock.ms(a, e) for a, _, e in marks), ws, device)
    solve_ms = max_over_ranks(sum(clock.ms(a, m) for a, m, _ in marks), ws, device)
    exch_ms = max_over_ranks(sum(clock.ms(m, e) for _, m, e in marks), ws, device)
    return {"job_ms": job, "solve_ms": solve_ms, "exchange_ms": exch_ms, "owned": owned, "bounds": b,
            "range": (lo, hi), "exchange": ex, "partial": partial, "solve_part": solve_part}


def sharded_same_split(offsets, nv, ws, partial_of):
    """The ws-way split run in one process (no collective): every range's partial from
    partial_of(lo, hi) -> (indptr, rows, values torch), combined in rank order by the owners as
    hyperalignment_b200.shard.exchange_in_process does.  The sharded run must equal it bit for bit."""
    from hyperalignment_b200 import shard as S
    import torch
    b = S.split_searchlights(offsets, ws)
    ptrs, rows, parts = [], [], []
    for q in range(ws):
        lo, hi = int(b[q]), int(b[q + 1])
        if hi > lo:
            p, r, v = partial_of(lo, hi)
        else:
            p, r, v = np.zeros(nv + 1, dtype=np.int64), np.zeros(0, dtype=np.int32), torch.zeros(0, dtype=torch.float64)
        ptrs.append(np.asarray(p, dtype=np.int64))
        rows.append(np.asarray(r, dtype=np.int32))
        parts.append(v)
    return S.exchange_in_process(ptrs, rows, parts, nv)


def bitwise_equal(a, b):
    return all(np.array_equal(np.asarray(x), np.asarray(y)) for x, y in zip(a, b))


def run_sharded_b200(args, ws, rank, local, lib):
    """bench.py --gpus N (N > 1): config 3's hemisphere (seed 0 on every rank) over the N GPUs with
    the tensor-core solver, one NCCL all-to-all of partial CSC values per step; value = searchlights
    of the hemisphere x steps / max over ranks of the device time (strong scaling).  Independent
    replicas (one hemisphere per GPU, no exchange) are a sub-field."""
    import torch
    import torch.distributed as dist
    from hyperalignment_b200 import _lib as L
    from hyperalignment_b200 import shard as S
    from hyperalignment_b200 import workloads as W
    from hyperalignment_b200.plan import Plan
    dev = torch.device("cuda", local)
    w3 = W.rank_deficient_pair(0, nv=args.nv, nt=args.nt)
    s = w3.sls
    K = args.steps
    hX = torch.from_numpy(np.asfortranarray(w3.X).ravel(order="F")).pin_memory()
    hY = torch.from_numpy(np.asfortranarray(w3.Y).ravel(order="F")).pin_memory()
    dX, dY = hX.to(dev), hY.to(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    wts = S.hemisphere_weights(s.indices, s.offsets, s.dists, s.radius, w3.nv)
    plans = []

    def make_range(lo, hi):
        idx, off, sw = S.sub_geometry(s.indices, s.offsets, wts, lo, hi)
        plan = Plan(w3.nt, w3.nv, idx, off, weights=sw)
        plans.append(plan)
        indptr, rows = plan.pattern()

        def solve(partial):
            plan.procrustes_device(dX.data_ptr(), dY.data_ptr(), partial.data_ptr(), True, True, L.SOLVER_TC,
                                   L.OUT_CSC, torch.cuda.current_stream(dev).cuda_stream)
        return indptr, rows, solve

    sampler = ClockSampler(local)
    sampler.start()
    n0 = lib.ha_b200_launch_count()
    res = sharded_rank(ws, rank, s.offsets, w3.nv, make_range, K, args.warmup, dev, flush=flush)
    launches = lib.ha_b200_launch_count() - n0
    clocks = sampler.stop()
    value = s.count * K / (res["job_ms"] / 1e3)
    ex = res["exchange"]

    # end to end: X and Y copied from pinned host memory, the owned values copied back, every step
    hout = torch.empty(res["owned"].numel(), dtype=torch.float64).pin_memory()
    stream = torch.cuda.current_stream(dev)
    for _ in range(args.warmup):
        dX.copy_(hX, non_blocking=True)
        dY.copy_(hY, non_blocking=True)
        res["solve_part"]()
        hout.copy_(ex.combine(res["partial"]), non_blocking=True)
    torch.cuda.synchronize()
    dist.barrier()
    ee = []
    for _ in range(K):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        dX.copy_(hX, non_blocking=True)
        dY.copy_(hY, non_blocking=True)
        res["solve_part"]()
        hout.copy_(ex.combine(res["partial"]), non_blocking=True)
        b.record(stream)
        ee.append((a, b))
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in ee), ws, dev)
    owned = ex.combine(res["partial"])
    full = ex.assemble(owned, dst=0)
    for p in plans:
        p.close()

    # replicas: every rank solves a whole hemisphere of its own (seed = rank), no exchange
    wr = W.rank_deficient_pair(rank, nv=args.nv, nt=args.nt)
    rplan = Plan.from_workload(wr)
    rX = torch.from_numpy(np.asfortranarray(wr.X).ravel(order="F")).to(dev)
    rY = torch.from_numpy(np.asfortranarray(wr.Y).ravel(order="F")).to(dev)
    rvals = torch.zeros(rplan.nnz, dtype=torch.float64, device=dev)

    def rstep():
        rplan.procrustes_device(rX.data_ptr(), rY.data_ptr(), rvals.data_ptr(), True, True, L.SOLVER_TC, L.OUT_CSR,
                                stream.cuda_stream)
    for _ in range(args.warmup):
        rstep()
    torch.cuda.synchronize()
    dist.barrier()
    evs = []
    for _ in range(K):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        rstep()
        b.record(stream)
        evs.append((a, b))
    torch.cuda.synchronize()
    rep_ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in evs), ws, dev)
    rplan.close()
    del rX, rY, rvals

    check = None
    if rank == 0:
        def partial_of(lo, hi):
            idx, off, sw = S.sub_geometry(s.indices, s.offsets, wts, lo, hi)
            plan = Plan(w3.nt, w3.nv, idx, off, weights=sw)
            v = torch.zeros(plan.nnz, dtype=torch.float64, device=dev)
            plan.procrustes_device(dX.data_ptr(), dY.data_ptr(), v.data_ptr(), True, True, L.SOLVER_TC, L.OUT_CSC,
                                   stream.cuda_stream)
            torch.cuda.synchronize()
            p, r = plan.pattern()
            plan.close()
            return p, r, v
        same = sharded_same_split(s.offsets, w3.nv, ws, partial_of)
        one = Plan.from_workload(w3)
        ref = torch.zeros(one.nnz, dtype=torch.float64, device=dev)
        one.procrustes_device(dX.data_ptr(), dY.data_ptr(), ref.data_ptr(), True, True, L.SOLVER_TC, L.OUT_CSC,
                              stream.cuda_stream)
        torch.cuda.synchronize()
        indptr, rows = one.pattern()
        refv = ref.cpu().numpy()
        one.close()
        pat = bool(np.array_equal(full[0], indptr) and np.array_equal(full[1], rows))
        check = {"bitwise_vs_same_split_on_rank0": bitwise_equal(full, same),
                 "pattern_identical_to_one_plan": pat,
                 "values_relfrob_vs_one_plan": float(np.linalg.norm(full[2] - refv) / np.linalg.norm(refv))
                 if pat else None,
                 "what": "the assembled CSC matrix against (a) the same N-way split solved on rank 0 and combined "
                         "in one process (must be bit-identical) and (b) one plan of the whole hemisphere (float64 "
                         "sums associated differently)"}
    dist.barrier()
    if rank == 0:
        lo, hi = res["range"]
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": K, "warmup": args.warmup,
            "ms_per_step": res["job_ms"] / K, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "tensor-core products, FP32-accurate splits: bf16x6 cross-covariance, fp16x3 iteration; f32/f64 host data", "data": "synthetic",
            "config": config_dict(w3, {"workload": WORKLOAD, "singular_searchlights": int(w3.extra["singular"].sum()),
                                       "parallelism": f"one hemisphere over {ws} GPUs: contiguous searchlight ranges "
                                                      "balanced by n^3, column owners, one NCCL all-to-all of partial "
                                                      "CSC values per step",
                                       "solver": "tensor cores: split-BF16 cross-covariance + split-FP16 Newton-Schulz polar"}),
            "solve_ms_per_step": res["solve_ms"] / K, "exchange_ms_per_step": res["exchange_ms"] / K,
            "searchlights_rank0": int(hi - lo), "columns_rank0": [int(c) for c in ex.col_range],
            "vs_one_plan": check,
            "replicas": {"value": aggregate_rate(ws, s.count, K, rep_ms / 1e3), "unit": UNIT, "ms_per_step": rep_ms / K,
                         "scaling": "weak", "what": "one hemisphere per GPU (seed = rank), no exchange"},
            "e2e": {"value": s.count * K / (e2e_ms / 1e3), "unit": UNIT,
                    "h2d_bytes_per_step": int(2 * w3.nt * w3.nv * 8), "d2h_bytes_per_step": int(hout.numel() * 8),
                    "path": "sharded step with X, Y copied from pinned host memory and the owned CSC values copied "
                            "back every step (rank 0's bytes)"},
            "roofline": None, "roofline_note": "reported by the one-GPU line",
            "cpu_baseline": None, "gpu_launches": int(launches), "clocks": clocks,
        }
        print(json.dumps(out))
    dist.barrier()
    dist.destroy_process_group()


def run_b200(args):
    import torch
    import torch.distributed as dist
    from hyperalignment_b200 import _lib as L
    from hyperalignment_b200 import workloads as W
    from hyperalignment_b200.plan import Plan

    ws, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    lib = L.lib()
    L.check(lib.ha_b200_init(), "ha_b200_init")
    if ws > 1:
        return run_sharded_b200(args, ws, rank, local, lib)

    # config 3 (headline): the template pair with ~10% of the searchlights made exactly singular;
    # config 2 (sub-field): the same pair without the duplicated columns
    w3 = W.rank_deficient_pair(rank, nv=args.nv, nt=args.nt)
    singular = w3.extra["singular"]
    w2 = workload(rank, args.nv, args.nt)
    assert np.array_equal(w2.Y, w3.Y) and np.array_equal(w2.sls.indices, w3.sls.indices)
    plan = Plan.from_workload(w3)
    dev = torch.device("cuda", local)
    dX3 = torch.from_numpy(np.asfortranarray(w3.X).ravel(order="F")).to(dev)
    dX2 = torch.from_numpy(np.asfortranarray(w2.X).ravel(order="F")).to(dev)
    dY = torch.from_numpy(np.asfortranarray(w3.Y).ravel(order="F")).to(dev)
    vals = torch.zeros(plan.nnz, dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step(solver, dX):
        plan.procrustes_device(dX.data_ptr(), dY.data_ptr(), vals.data_ptr(), True, True, solver, L.OUT_CSR,
                               stream.cuda_stream)

    def timed_loop(solver, dX, k, sample_clocks=False, trace=False):
        for _ in range(args.warmup):
            step(solver, dX)
        torch.cuda.synchronize()
        if ws > 1:
            dist.barrier()
        sampler = ClockSampler(local) if sample_clocks else None
        if sampler:
            sampler.start()
            time.sleep(0.5)
        if trace:
            lib.ha_b200_kernel_times(None, None)
            lib.ha_b200_set_kernel_timing(True)
        n0 = lib.ha_b200_launch_count()
        torch.cuda.synchronize()
        evs = []
        t0 = time.perf_counter()
        for _ in range(k):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            step(solver, dX)
            b.record(stream)
            evs.append((a, b))
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        launches = lib.ha_b200_launch_count() - n0
        kt = None
        if trace:
            lib.ha_b200_set_kernel_timing(False)
            ms = np.zeros(len(L.KERNEL_KINDS))
            cnt = np.zeros(len(L.KERNEL_KINDS), dtype=np.int64)
            lib.ha_b200_kernel_times(ms.ctypes.data_as(L.c_double_p), cnt.ctypes.data_as(L.c_int64_p))
            kt = (ms, cnt)
        clocks = sampler.stop() if sampler else None
        dev_ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in evs), ws, dev)
        if ws > 1:
            dist.barrier()
        return dev_ms, wall, launches, kt, clocks

    K = args.steps
    count = w3.sls.count
    # untimed iteration counts of the tensor-core solve (for the roofline's work per launch)
    step(L.SOLVER_TC, dX3)
    torch.cuda.synchronize()
    tc_iters = plan.searchlight_stats(0, count)["sweeps"].astype(np.int64)
    tc_flags = plan.searchlight_stats(0, count)["flags"]
    # the value: untraced (the iteration replays as a CUDA graph, no per-launch events)
    total_ms, wall, launches, _, clocks = timed_loop(L.SOLVER_TC, dX3, K, sample_clocks=True)
    value = aggregate_rate(ws, count, K, total_ms / 1e3)
    tc_stats = plan.stats()
    tc_layout = plan.tc_layout()
    # per-kind kernel times from separate traced steps (CUDA events around every launch)
    KT = max(2, K // 3)
    traced_ms, _, _, kt, _ = timed_loop(L.SOLVER_TC, dX3, KT, trace=True)
    plain_ms, _, _, _, _ = timed_loop(L.SOLVER_FP32, dX3, K)
    plain_value = aggregate_rate(ws, count, K, plain_ms / 1e3)
    plain_stats = plan.stats()
    km = max(1, K // 2)
    mixed_ms, _, _, _, _ = timed_loop(L.SOLVER_MIXED, dX3, km)
    mixed_value = aggregate_rate(ws, count, km, mixed_ms / 1e3)
    mixed_stats = plan.stats()
    fp64_ms, _, _, _, _ = timed_loop(L.SOLVER_FP64, dX3, 1)
    fp64_value = aggregate_rate(ws, count, 1, fp64_ms / 1e3)
    # config 2: the same step without the duplicated columns
    c2_ms, _, _, _, _ = timed_loop(L.SOLVER_TC, dX2, K)
    c2_value = aggregate_rate(ws, count, K, c2_ms / 1e3)
    c2_stats = plan.stats()
    c2_plain_ms, _, _, _, _ = timed_loop(L.SOLVER_FP32, dX2, K)
    c2_plain = aggregate_rate(ws, count, K, c2_plain_ms / 1e3)

    # accuracy vs the float64 oracle on fixed samples (24 singular + 24 regular searchlights of
    # config 3, 24 of config 2), solved by a plan over the sampled searchlights only (same kernels)
    rng = np.random.default_rng(7)
    sing, reg = np.flatnonzero(singular), np.flatnonzero(~singular)
    sample3 = np.sort(np.concatenate([rng.choice(sing, size=min(24, sing.size), replace=False),
                                      rng.choice(reg, size=min(24, reg.size), replace=False)]))
    sample2 = np.sort(np.random.default_rng(123).choice(count, size=24, replace=False))
    errs, errs2 = {}, {}
    for smp, wk, dX, sg, out in ((sample3, w3, dX3, singular, errs), (sample2, w2, dX2, None, errs2)):
        sub = wk.sls.subset(smp)
        splan = Plan(wk.nt, wk.nv, sub.indices, sub.offsets, sub.dists, sub.radius)
        svals = torch.zeros(splan.nnz, dtype=torch.float64, device=dev)
        for name, solver in (("tensor_core", L.SOLVER_TC), ("plain_fp32", L.SOLVER_FP32), ("mixed", L.SOLVER_MIXED)):
            splan.procrustes_device(dX.data_ptr(), dY.data_ptr(), svals.data_ptr(), True, True, solver, L.OUT_CSR,
                                    stream.cuda_stream)
            torch.cuda.synchronize()
            out[name] = sample_errors(wk, sg, smp, splan.local_transforms(0, sub.count))
        splan.close()

    # roofline of the dominant kernel (the Newton-Schulz products on the tensor cores)
    peaks, peak_src = load_peaks()
    ms, cnt = kt
    dom = int(np.argmax(ms))
    dom_name = L.KERNEL_KINDS[dom]
    sizes = w3.sls.sizes
    roof = None
    if dom_name == "tc_ns" and ms[dom] > 0:
        per_step = tc_algorithmic_flops(sizes, tc_iters)
        per_launch = per_step * KT / max(1, cnt[dom])
        avg_ms = ms[dom] / max(1, cnt[dom])
        achieved = per_launch / (avg_ms / 1e3)
        peak = float(peaks.get("bf16_tflops_sustained", peaks.get("bf16_tflops")))
        executed = tc_executed_flops(sizes, tc_iters) * KT / max(1, cnt[dom]) / (avg_ms / 1e3)
        useful = 23.0 * float((sizes.astype(np.float64) ** 3).sum()) * KT / max(1, cnt[dom]) / (avg_ms / 1e3)
        roof = {"bound": "tensor", "kernel": "tc_ns (k_tc_gemm Gram + update, k_tc_ns_init)", "achieved": achieved / 1e12,
                "peak": peak, "unit": "TFLOP/s", "frac": achieved / 1e12 / peak, "traffic": None,
                "peak_source": f"{peak_src} bf16 sustained",
                "algorithmic": "12 n^3 tensor flops per searchlight and iteration (two n^3 products, three FP16 "
                               "products each); iterations as run (mean %.2f)" % float(tc_iters.mean()),
                "executed_with_padding_tflops": executed / 1e12,
                "svd_equivalent_tflops": useful / 1e12,
                "svd_equivalent": "23 n^3 per searchlight (square SVD 21 n^3 + U V^T 2 n^3, the reference's work)",
                "avg_launch_ms": float(avg_ms), "launches_per_step": float(cnt[dom] / KT),
                "timing": f"{KT} separate traced steps (CUDA events around every launch, no graph replay): "
                          f"{traced_ms / KT:.2f} ms per step against {total_ms / K:.2f} untraced"}
    elif ms[dom] > 0:
        roof = {"bound": "unknown", "kernel": dom_name, "achieved": None, "peak": None, "unit": None, "frac": None,
                "traffic": None}
    traffic_file = os.path.join(ROOT, "profiles", "traffic.json")
    if roof is not None and os.path.exists(traffic_file):
        with open(traffic_file) as f:
            tr = json.load(f)
        if dom_name in tr:
            per_sl = tr[dom_name].get("bytes_per_searchlight")
            if per_sl:
                # ncu capture of a smaller case scaled to a full launch by the searchlights it solves
                roof["traffic"] = per_sl * count * KT / max(1, cnt[dom])
                roof["traffic_source"] = tr[dom_name].get("source")
    kernel_share = {L.KERNEL_KINDS[i]: {"ms_per_step": float(ms[i] / KT), "launches_per_step": float(cnt[i] / KT)}
                    for i in range(len(ms)) if cnt[i] > 0}

    # end to end through the C ABI dense entry point (host buffers): warm calls, then one cold call
    # after ha_b200_cleanup (plan, pattern and buffers rebuilt, as a caller that cleans up after
    # every call pays)
    e2e = None
    if not args.no_e2e:
        Xf, Yf = np.asfortranarray(w3.X), np.asfortranarray(w3.Y)
        T_out = np.zeros((w3.nv, w3.nv))
        s = w3.sls
        argsv = (Xf.ctypes.data_as(L.c_double_p), Yf.ctypes.data_as(L.c_double_p), w3.nt, w3.nv,
                 L.iptr(s.indices), L.iptr(s.offsets), L.dptr(s.dists), s.count, s.radius,
                 T_out.ctypes.data_as(L.c_double_p), True, True, L.BACKEND_B200, True)
        lib.ha_set_num_threads(os.cpu_count() or 1)
        for _ in range(max(1, args.warmup)):
            L.check(lib.ha_searchlight_procrustes_dense(*argsv), "dense")
        if ws > 1:
            dist.barrier()
        ts = []
        for _ in range(K):
            t0 = time.perf_counter()
            L.check(lib.ha_searchlight_procrustes_dense(*argsv), "dense")
            ts.append(time.perf_counter() - t0)
        tmax = max_over_ranks(sum(ts), ws, dev)
        lib.ha_b200_cleanup()
        t0 = time.perf_counter()
        L.check(lib.ha_searchlight_procrustes_dense(*argsv), "dense")
        cold = max_over_ranks(time.perf_counter() - t0, ws, dev)
        e2e = {"value": aggregate_rate(ws, s.count, K, tmax), "unit": UNIT,
               "h2d_bytes_per_step": int(2 * w3.nt * w3.nv * 8), "d2h_bytes_per_step": int(plan.nnz * 8),
               "path": "ha_searchlight_procrustes_dense(backend=4) host float64 in, host dense nv x nv out (+=); "
                       "tensor-core solver",
               "cold_first_call": {"value": aggregate_rate(ws, s.count, 1, cold), "unit": UNIT, "seconds": cold,
                                   "what": "first call after ha_b200_cleanup: plan, pattern, work lists and "
                                           "buffers built inside the call"}}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        from oracle import ref_lib as R
        if R.available():
            threads = os.cpu_count() or 1
            r, m, dt = reference_rate(w3, args.cpu_seconds, threads)
            r1, m1, dt1 = reference_rate(w3, min(5.0, args.cpu_seconds / 3.0), 1)
            r32, m32, dt32 = reference_rate(w3, min(5.0, args.cpu_seconds / 3.0), threads, backend=1)
            cpu = {"value": r, "unit": UNIT, "cores": threads, "kind": "reference",
                   "sample": f"{m} contiguous searchlights of {count} ({dt:.1f} s), reference cpu64 arm, "
                             f"OpenMP {threads} threads, OPENBLAS_NUM_THREADS=1",
                   "single_thread": {"value": r1, "unit": UNIT, "cores": 1,
                                     "sample": f"{m1} contiguous searchlights ({dt1:.1f} s), one OpenMP thread"},
                   "cpu32_arm": {"value": r32, "unit": UNIT, "cores": threads,
                                 "sample": f"{m32} contiguous searchlights ({dt32:.1f} s), the reference's float32 "
                                           f"arm, OpenMP {threads} threads"}}
        else:
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                   "sample": "oracle/_ref/libhyperalignment.so not built"}

    # configs 4 and 5 (the grid search at full size, the learned proposal), after the headline's
    # timed steps; a failure there is reported in its field and does not lose the line
    extras = {}
    if not args.no_extras:
        plan.close()
        for key, fn in (("config4_ridge_grid_full", lambda: config4_grid_full(args, dev)),
                        ("config5_learned", lambda: config5_learned(args))):
            try:
                extras[key] = fn()
            except Exception as ex:  # noqa: BLE001
                extras[key] = {"error": repr(ex)}

    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": K, "warmup": args.warmup,
            "ms_per_step": total_ms / K, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "tensor-core products, FP32-accurate splits: bf16x6 cross-covariance, fp16x3 iteration; f32/f64 host data", "data": "synthetic",
            "config": config_dict(w3, {"workload": WORKLOAD, "singular_searchlights": int(singular.sum()),
                                       "parallelism": "single GPU (bench.py --gpus N shards this hemisphere over N)",
                                       "solver": "tensor cores: split-BF16 cross-covariance + split-FP16 Newton-Schulz polar, "
                                                 "null-space completion of exactly singular searchlights"}),
            "plain_fp32": {"value": plain_value, "unit": UNIT, "ms_per_step": plain_ms / K,
                           "speedup_of_value": value / plain_value, "what": "FP32 Jacobi SVD, no refinement, no FP64"},
            "mixed_form": {"value": mixed_value, "unit": UNIT, "ms_per_step": mixed_ms / km,
                           "what": "FP32 Jacobi + Newton-Schulz refinement + FP64 re-solve below sigma ratio 5e-5"},
            "fp64_form": {"value": fp64_value, "unit": UNIT},
            "config2_template_pair": {"value": c2_value, "unit": UNIT, "ms_per_step": c2_ms / K,
                                      "plain_fp32": c2_plain, "speedup_of_value": c2_value / c2_plain,
                                      "solver_stats": c2_stats, "error_vs_fp64": errs2},
            "error_vs_fp64": errs,
            "solver_stats": {"tensor_core": tc_stats, "plain_fp32": plain_stats, "mixed": mixed_stats,
                             "completed_null_spaces": int(((tc_flags & 16) != 0).sum()),
                             "tc_layout": tc_layout,
                             "iterations_mean": float(tc_iters.mean()), "iterations_max": int(tc_iters.max())},
            "roofline": roof,
            "kernels": kernel_share,
            "kernels_note": "per-kind CUDA-event intervals of separate traced tensor-core steps; its kernels run in "
                            "order on one stream (the float64 re-solve's side streams run only for searchlights left "
                            "flagged)",
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": int(launches),
            "clocks": clocks,
            "wall_s_timed": wall,
            **extras,
        }
        print(json.dumps(out))
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()


# ---------------------------------------------------------------------------------------------
# the reference's own GPU arm on the same B200 (its cuBLAS + cuSOLVER path, rebuilt for sm_100a)
# ---------------------------------------------------------------------------------------------

def run_refgpu(args):
    """Config 1 (2562 vertices, nt 200, geodesic-disc searchlights of 71-78, reflection allowed, no
    scaling) and the Forrest shape (9675 vertices, nt 1818, searchlights of 90-170): the reference's
    CUDA arm (dense entry, backend 3) against this library's tensor-core solver and its plain FP32
    form, all from host buffers into a host dense nv x nv matrix, wall clock per call; errors of the
    dense result against the reference's float64 CPU arm."""
    import torch
    from hyperalignment_b200 import _lib as L
    from hyperalignment_b200 import workloads as W
    from hyperalignment_b200.plan import Plan
    from oracle import ref_lib as R

    ws, rank, local = dist_setup(args)
    if rank != 0:
        return
    torch.cuda.set_device(local)
    lib = L.lib()
    L.check(lib.ha_b200_init(), "ha_b200_init")
    if not R.cuda_available():
        print(json.dumps({"workload": "refgpu", "unavailable": "oracle/_ref_cuda not built (make -C oracle cuda)"}))
        return
    rc_lib = R.cuda_lib()
    if rc_lib.ha_cuda_init() != 0 or not rc_lib.ha_cuda_available():
        print(json.dumps({"workload": "refgpu", "unavailable": "the reference's ha_cuda_init failed on this GPU"}))
        return
    rc_lib.ha_set_num_threads(os.cpu_count() or 1)
    R.set_threads(os.cpu_count() or 1)
    out = {"workload": "reference_gpu_comparison", "unit": UNIT, "higher_is_better": True, "data": "synthetic",
           "path": "host float64 in, host dense nv x nv float64 out, wall clock per call", "configs": {}}
    for name, w in (("config1_plain_procrustes", W.plain_procrustes(0)), ("forrest_shaped", W.forrest_shaped(0))):
        s = w.sls
        Xf, Yf = np.asfortranarray(w.X), np.asfortranarray(w.Y)
        nt, nv = w.nt, w.nv
        ref64 = R.procrustes_dense(w.X, w.Y, s.indices, s.offsets, s.dists, s.radius, True, False, 0)
        nref = np.linalg.norm(ref64)

        def err(T):
            """Relative Frobenius and max-abs error over the finite entries, and how many are not finite
            (the reference's CUDA arm does not check cuSOLVER's per-matrix status)."""
            ok = np.isfinite(T)
            d = np.where(ok, T - ref64, 0.0)
            bad = np.flatnonzero(~ok.all(axis=1))
            return {"relfrob": float(np.linalg.norm(d) / nref), "maxabs": float(np.abs(d).max()),
                    "nonfinite_entries": int((~ok).sum()), "rows_with_nonfinite": int(bad.size)}

        def time_calls(call, k):
            call()
            ts = []
            for _ in range(k):
                t0 = time.perf_counter()
                call()
                ts.append(time.perf_counter() - t0)
            return s.count * k / sum(ts), float(np.mean(ts))

        T_ref = np.zeros((nv, nv))

        def ref_call():
            T_ref[:] = 0.0
            rc = rc_lib.ha_searchlight_procrustes_dense(
                Xf.ctypes.data_as(R.c_double_p), Yf.ctypes.data_as(R.c_double_p), nt, nv,
                s.indices.ctypes.data_as(R.c_int32_p), s.offsets.ctypes.data_as(R.c_int32_p),
                s.dists.ctypes.data_as(R.c_double_p), s.count, s.radius, T_ref.ctypes.data_as(R.c_double_p),
                True, False, 3, True)
            if rc != 0:
                raise RuntimeError(f"reference CUDA rc={rc}")

        k_ref = max(1, min(args.steps, 3))
        r_val, r_s = time_calls(ref_call, k_ref)
        T_tc = np.zeros((nv, nv))
        argsv = (Xf.ctypes.data_as(L.c_double_p), Yf.ctypes.data_as(L.c_double_p), nt, nv, L.iptr(s.indices),
                 L.iptr(s.offsets), L.dptr(s.dists), s.count, s.radius, T_tc.ctypes.data_as(L.c_double_p),
                 True, False, L.BACKEND_B200, True)

        def tc_call():
            T_tc[:] = 0.0
            L.check(lib.ha_searchlight_procrustes_dense(*argsv), "dense")

        t_val, t_s = time_calls(tc_call, max(1, min(args.steps, 5)))
        # plain FP32 form of this library on device-resident inputs (the metric's denominator)
        plan = Plan.from_workload(w)
        dX = torch.from_numpy(np.asfortranarray(w.X).ravel(order="F")).cuda()
        dY = torch.from_numpy(np.asfortranarray(w.Y).ravel(order="F")).cuda()
        vals = torch.zeros(plan.nnz, dtype=torch.float64, device="cuda")
        evs = []
        for i in range(4):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            plan.procrustes_device(dX.data_ptr(), dY.data_ptr(), vals.data_ptr(), True, False, L.SOLVER_FP32,
                                   L.OUT_CSR)
            b.record()
            evs.append((a, b))
        torch.cuda.synchronize()
        p_ms = min(a.elapsed_time(b) for a, b in evs[1:])
        plan.close()
        sizes = s.sizes
        out["configs"][name] = {
            "nv": nv, "nt": nt, "searchlights": s.count, "sl_size_min": int(sizes.min()),
            "sl_size_max": int(sizes.max()), "reflection": True, "scaling": False,
            "reference_cuda": {"value": r_val, "seconds_per_call": r_s, "calls": k_ref, "error_vs_cpu64": err(T_ref),
                               "what": "reference csrc/ha_cuda.cu (cuBLAS SGEMM batched + cuSOLVER "
                                       "gesvdaStridedBatched, batches of 256 padded to max_sz), -arch sm_100a"},
            "tensor_core": {"value": t_val, "seconds_per_call": t_s, "error_vs_cpu64": err(T_tc),
                            "what": "ha_searchlight_procrustes_dense(backend=4), tensor-core solver"},
            "speedup_vs_reference_cuda": t_val / r_val,
            "plain_fp32_device": {"value": s.count / (p_ms / 1e3), "ms": p_ms},
        }
    rc_lib.ha_cuda_cleanup()
    print(json.dumps(out))


# ---------------------------------------------------------------------------------------------
# ridge grid search (40962 vertices, sizes 50-500, nt 500, 10 alphas x 4 PC counts, 5 CV folds)
# and the learned proposal on top of it
# ---------------------------------------------------------------------------------------------

FP64_NOMINAL_TFLOPS = 37.0  # B200 float64 (context only; the kernels run on the FP64 SIMT pipe)


def _oracle_grid_worker(args):
    import os as _os
    _os.environ["OPENBLAS_NUM_THREADS"] = "1"
    X, Y, sl, alphas, npcs, tr, te = args
    from oracle import ha_oracle as O
    O.ensemble_ridge(X[:, sl], Y[:, sl], alphas, npcs, tr, te)
    return sl.size


def grid_cpu_rate(w, sls, tr, te, seconds):
    """The oracle's composition (numpy, one BLAS thread per process, all host cores) on the first
    searchlights of the subset, sized to about ``seconds``."""
    import multiprocessing as mp
    from hyperalignment_b200 import workloads as W
    cores = os.cpu_count() or 1
    m = max(cores, int(seconds * cores / 1.3))
    m = min(m, sls.count)
    jobs = []
    for q in range(m):
        sl = sls.indices[sls.offsets[q]:sls.offsets[q + 1]]
        jobs.append((np.ascontiguousarray(w.X[:, sl]), np.ascontiguousarray(w.Y[:, sl]), np.arange(sl.size),
                     W.GRID_ALPHAS, W.GRID_NPCS, tr, te))
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        t0 = time.perf_counter()
        pool.map(_oracle_grid_worker, jobs, chunksize=1)
        dt = time.perf_counter() - t0
    return m / dt, m, dt, cores


def config4_grid_full(args, dev):
    """Config 4 at full size, a sub-field of the default line: the ridge grid search (10 alphas x
    4 PC counts, 5-fold blocked CV with 10-TR buffers) over all 40962 searchlights of 50-500
    vertices, nt 500, AR(1) noise; one warm-up and one timed step (CUDA events, L2 flushed).  The
    winners and cost grids of a sample of searchlights are checked against the oracle's
    composition of ha_ensemble_ridge."""
    import torch
    from hyperalignment_b200 import hyperalignment_c as H
    from hyperalignment_b200 import workloads as W
    from hyperalignment_b200.plan import Plan
    from oracle import ha_oracle as O
    w = W.ridge_grid_pair(0, nv=40962, nt=500)
    sls = w.sls
    tr, te = H.ensemble_indices(w.nt, 1, 5, 10, 10, 0)
    plan = Plan(w.nt, w.nv, sls.indices, sls.offsets, sls.dists, sls.radius)
    dX = torch.from_numpy(np.asfortranarray(w.X).ravel(order="F")).to(dev)
    dY = torch.from_numpy(np.asfortranarray(w.Y).ravel(order="F")).to(dev)
    vals = torch.zeros(plan.nnz, dtype=torch.float64, device=dev)
    best = torch.zeros(sls.count, dtype=torch.int32, device=dev)
    grid = len(W.GRID_ALPHAS) * len(W.GRID_NPCS)
    cost = torch.zeros(sls.count * grid, dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step():
        vals.zero_()
        plan.ridge_grid_device(dX.data_ptr(), dY.data_ptr(), vals.data_ptr(), best.data_ptr(), W.GRID_ALPHAS,
                               W.GRID_NPCS, tr, te, d_cost=cost.data_ptr(), stream=stream.cuda_stream)

    t0 = time.perf_counter()
    step()  # warm-up: plan work lists, graph capture
    torch.cuda.synchronize()
    first_s = time.perf_counter() - t0
    flush.zero_()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    step()
    b.record(stream)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b)
    hb, hc = best.cpu().numpy(), cost.cpu().numpy().reshape(sls.count, grid)
    rng = np.random.default_rng(4)
    sample = np.sort(rng.choice(sls.count, 6, replace=False))
    rel, same = [], 0
    for q in sample:
        sl = sls.indices[sls.offsets[q]:sls.offsets[q + 1]]
        r = O.ensemble_ridge(w.X[:, sl], w.Y[:, sl], W.GRID_ALPHAS, W.GRID_NPCS, tr, te)
        rc = np.asarray(r[6]).ravel()
        rel.append(float(np.max(np.abs(hc[q] - rc) / np.abs(rc))))
        same += int(hb[q] == int(np.argmin(rc)))
    # the plain FP32 form of the same grid search: one warm-up, one timed step, costs and winners
    # against the float64 search's (all searchlights)
    plan.set_grid_precision(32)
    best32 = torch.zeros_like(best)
    cost32 = torch.zeros_like(cost)

    def step32():
        vals.zero_()
        plan.ridge_grid_device(dX.data_ptr(), dY.data_ptr(), vals.data_ptr(), best32.data_ptr(), W.GRID_ALPHAS,
                               W.GRID_NPCS, tr, te, d_cost=cost32.data_ptr(), stream=stream.cuda_stream)

    step32()
    torch.cuda.synchronize()
    flush.zero_()
    a.record(stream)
    step32()
    b.record(stream)
    torch.cuda.synchronize()
    ms32 = a.elapsed_time(b)
    plan.set_grid_precision(64)
    hb32, hc32 = best32.cpu().numpy(), cost32.cpu().numpy().reshape(sls.count, grid)
    rows = np.arange(sls.count)
    plain = {"value": sls.count / (ms32 / 1e3), "ms_per_step": ms32, "steps": 1, "warmup": 1, "dtype": "f32",
             "cost_grid_max_rel_vs_f64": float(np.max(np.abs(hc32 - hc) / np.abs(hc))),
             "winners_equal_f64": float(np.mean(hb32 == hb)),
             "winner_cost_regret_max": float(np.max(hc[rows, hb32] / hc.min(axis=1) - 1.0))}
    st = plan.stats()
    plan.close()
    sizes = sls.sizes
    return {"value": sls.count / (ms / 1e3), "unit": UNIT, "ms_per_step": ms, "steps": 1, "warmup": 1,
            "plain_fp32": plain, "speedup_over_plain_fp32": ms32 / ms,
            "first_call_s": first_s,
            "config": {"workload": "ridge_grid_full", "nv": w.nv, "nt": w.nt, "searchlights": sls.count,
                       "sl_size_min": int(sizes.min()), "sl_size_max": int(sizes.max()),
                       "alphas": "10 log-spaced in [1e-3, 1e3]", "npcs": [10, 20, 50, "all"],
                       "cv": "ha_ensemble_indices(500, 1, 5, 10, 10, 0)", "noise": "AR(1) rho 0.5",
                       "dtype": "f64", "l2": "flushed before the timed step"},
            "error_vs_oracle": {"cost_grid_max_rel": max(rel), "winners_identical": f"{same} of {len(sample)}",
                                "sample": [int(q) for q in sample]},
            "winners_distinct": int(np.unique(hb).size), "solver_stats": st}


def config5_learned(args):
    """Config 5, a sub-field of the default line: the learned (alpha, PC count) proposal on the
    40962-vertex grid workload.  The perceptron is trained on the GPU on the full grid's winners for
    four training subjects (every 16th searchlight each), then the held-out subject (every 4th
    searchlight, 10240) runs through the full grid and through the learned form (proposal where its
    probability is at least 0.6, the full grid elsewhere); warm runs are timed.  The value is the
    mixed-precision learned form (float32 eigen solve, proposal fit and fallback grid, bf16
    inference), set against the plain FP32 full grid on the same searchlights; the float64 full grid
    and the float64 learned form are sub-fields.  The generator's noise
    amplitude varies from 0.2 to 6 over the sphere so that the best grid point varies between
    searchlights (with homogeneous noise one grid point wins almost everywhere)."""
    from hyperalignment_b200 import learned as LR
    res = LR.study(nv=40962, step=4, train_step=16, size_lo=50, size_hi=500, epochs=60, log=lambda *a: None)
    g, l, g32, m = res["grid"], res["learned"], res["grid_fp32"], res["learned_fp32"]
    return {"value": m["searchlights_per_s"], "unit": UNIT, "ms_per_step": m["ms"],
            "form": "mixed-precision learned form: float32 eigen solve, features, proposal fit and fallback grid; "
                    "bf16 inference; float64 inputs, betas and reduction",
            "plain_fp32_grid": {"value": g32["searchlights_per_s"], "ms_per_step": g32["ms"],
                                "heldout_corr": g32["heldout_corr"], "winners_equal_fp64": g32["winners_equal_fp64"]},
            "speedup_over_plain_fp32_grid": m["searchlights_per_s"] / g32["searchlights_per_s"],
            "heldout_corr": m["heldout_corr"], "heldout_corr_minus_plain_fp32_grid": m["heldout_corr"] - g32["heldout_corr"],
            "fallback_searchlights": m["fallback"], "choices_equal_fp64_learned": m["choices_equal_fp64_learned"],
            "full_grid": {"value": g["searchlights_per_s"], "ms_per_step": g["ms"], "heldout_corr": g["heldout_corr"]},
            "learned_fp64": {"value": l["searchlights_per_s"], "ms_per_step": l["ms"], "heldout_corr": l["heldout_corr"],
                             "fallback_searchlights": l["fallback"],
                             "speedup_over_full_grid": l["searchlights_per_s"] / g["searchlights_per_s"]},
            "heldout_corr_minus_grid": m["heldout_corr"] - g["heldout_corr"],
            "proposal_matches_grid": l["proposal_matches_grid"],
            "fixed_point": res["fixed_point"], "train": res["train"],
            "config": {"workload": "ridge_grid_learned", "nv": 40962, "nt": 500, "fit_rows": 400, "eval_rows": 100,
                       "heldout_searchlights": res["searchlights"], "train_subset": "every 16th, seeds 1-4",
                       "heldout_subset": "every 4th, seed 5", "sizes": "50-500",
                       "noise": "AR(1) rho 0.5, amplitude 0.2 to 6 over the sphere", "min_prob": 0.6}}


def run_grid(args):
    import torch
    from hyperalignment_b200 import _lib as L
    from hyperalignment_b200 import hyperalignment_c as H
    from hyperalignment_b200 import workloads as W
    from hyperalignment_b200.plan import Plan

    ws, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    lib = L.lib()
    L.check(lib.ha_b200_init(), "ha_b200_init")
    nv = 40962 if args.nv == 10242 else args.nv
    w = W.ridge_grid_pair(rank, nv=nv, nt=500)
    sls = w.sls.subset(np.arange(0, w.sls.count, args.grid_step))
    tr, te = H.ensemble_indices(w.nt, 1, 5, 10, 10, rank)
    plan = Plan(w.nt, w.nv, sls.indices, sls.offsets, sls.dists, sls.radius)
    plan.set_grid_precision(args.grid_bits)
    dev = torch.device("cuda", local)
    dX = torch.from_numpy(np.asfortranarray(w.X).ravel(order="F")).to(dev)
    dY = torch.from_numpy(np.asfortranarray(w.Y).ravel(order="F")).to(dev)
    vals = torch.zeros(plan.nnz, dtype=torch.float64, device=dev)
    best = torch.zeros(sls.count, dtype=torch.int32, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step():
        plan.ridge_grid_device(dX.data_ptr(), dY.data_ptr(), vals.data_ptr(), best.data_ptr(), W.GRID_ALPHAS,
                               W.GRID_NPCS, tr, te, stream=stream.cuda_stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    K = args.steps
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.5)
    lib.ha_b200_kernel_times(None, None)
    lib.ha_b200_set_kernel_timing(True)
    n0 = lib.ha_b200_launch_count()
    evs = []
    t0 = time.perf_counter()
    for _ in range(K):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        step()
        b.record(stream)
        evs.append((a, b))
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    launches = lib.ha_b200_launch_count() - n0
    lib.ha_b200_set_kernel_timing(False)
    ms = np.zeros(len(L.KERNEL_KINDS))
    cnt = np.zeros(len(L.KERNEL_KINDS), dtype=np.int64)
    lib.ha_b200_kernel_times(ms.ctypes.data_as(L.c_double_p), cnt.ctypes.data_as(L.c_int64_p))
    clocks = sampler.stop()
    total_ms = float(sum(a.elapsed_time(b) for a, b in evs))
    value = sls.count * K / (total_ms / 1e3)
    st = plan.stats()

    # roofline of the dominant kernel: the float64 Jacobi eigen solves (9 n^3 flops per
    # symmetric eigendecomposition with vectors, Golub-Van Loan count; 5 CV models per searchlight)
    peaks, peak_src = load_peaks()
    dom = int(np.argmax(ms))
    n3 = float((sls.sizes.astype(np.float64) ** 3).sum())
    roof = None
    if L.KERNEL_KINDS[dom] in ("jacobi64", "jacobi32") and ms[dom] > 0:
        achieved = 9.0 * n3 * len(tr) * K / (ms[dom] / 1e3) / 1e12
        peak = float(peaks.get("bf16_tflops_sustained", peaks.get("bf16_tflops")))
        roof = {"bound": "tensor", "kernel": f"{L.KERNEL_KINDS[dom]} (eigenvector mode)", "achieved": achieved, "peak": peak,
                "unit": "TFLOP/s", "frac": achieved / peak, "traffic": None,
                "peak_source": f"{peak_src} bf16 sustained",
                "fp64_simt": {"peak_nominal": FP64_NOMINAL_TFLOPS, "frac": achieved / FP64_NOMINAL_TFLOPS},
                "algorithmic": "9 n^3 flops per symmetric eigendecomposition, 5 per searchlight"}

    # end to end through the host C ABI entry (host float64 in, host CSC values out)
    e2e = None
    if not args.no_e2e:
        indptr, indices = plan.pattern()
        ip32, ind32 = indptr.astype(np.int32), indices.astype(np.int32)
        sl_lists = [sls.indices[sls.offsets[q]:sls.offsets[q + 1]] for q in range(sls.count)]
        wts = H.searchlight_weights(sl_lists, [sls.dists[sls.offsets[q]:sls.offsets[q + 1]] for q in range(sls.count)],
                                    sls.radius, w.nv)
        data = np.zeros(indices.size)
        H.searchlight_ridge_grid(w.X, w.Y, sl_lists, ip32, ind32, data, W.GRID_ALPHAS, W.GRID_NPCS, tr, te,
                                 weights=[wts])
        ts = []
        for _ in range(K):
            data[:] = 0.0
            t1 = time.perf_counter()
            H.searchlight_ridge_grid(w.X, w.Y, sl_lists, ip32, ind32, data, W.GRID_ALPHAS, W.GRID_NPCS, tr, te,
                                     weights=[wts])
            ts.append(time.perf_counter() - t1)
        e2e = {"value": sls.count * K / sum(ts), "unit": UNIT, "h2d_bytes_per_step": int(2 * w.nt * w.nv * 8),
               "d2h_bytes_per_step": int(plan.nnz * 8 + sls.count * 4),
               "path": "ha_searchlight_ridge_grid_b200 host float64 in, host CSC values out (+=)"
                       + ("; the host entry is float64 whatever --grid-bits" if args.grid_bits == 32 else "")}

    cpu = None
    if rank == 0 and not args.no_cpu:
        r, m, dt, cores = grid_cpu_rate(w, sls, tr, te, args.cpu_seconds)
        cpu = {"value": r, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"{m} searchlights of the subset ({dt:.1f} s), oracle composition of ha_ensemble_ridge "
                         f"(numpy, one BLAS thread per process, {cores} processes)"}
    if rank == 0:
        sizes = sls.sizes
        out = {"metric": "searchlight ridge grid searches/sec", "value": value, "unit": UNIT, "n_gpus": 1,
               "steps": K, "warmup": args.warmup, "ms_per_step": total_ms / K, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.grid_bits == 64 else "f32",
               "data": "synthetic",
               "config": {"workload": "ridge_grid", "nv": w.nv, "nt": w.nt, "searchlights": sls.count,
                          "searchlight_subset": f"every {args.grid_step}th of {w.sls.count}",
                          "sl_size_min": int(sizes.min()), "sl_size_max": int(sizes.max()),
                          "sl_size_mean": round(float(sizes.mean()), 2), "alphas": "10 log-spaced in [1e-3, 1e3]",
                          "npcs": [10, 20, 50, "all"], "cv": "ha_ensemble_indices(500, 1, 5, 10, 10, seed)",
                          "noise": "AR(1) rho 0.5", "l2": "flushed between steps (256 MiB write)"},
               "solver_stats": st, "winners_distinct": int(np.unique(best.cpu().numpy()).size),
               "roofline": roof,
               "kernels": {L.KERNEL_KINDS[i]: {"ms_per_step": float(ms[i] / K), "launches_per_step": float(cnt[i] / K)}
                           for i in range(len(ms)) if cnt[i] > 0},
               "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches), "clocks": clocks,
               "wall_s_timed": wall}
        print(json.dumps(out))


def run_learned(args):
    import torch
    from hyperalignment_b200 import _lib as L
    from hyperalignment_b200 import learned as LR

    ws, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    L.check(L.lib().ha_b200_init(), "ha_b200_init")
    nv = args.nv
    res = LR.study(nv=nv, step=4, size_lo=50, size_hi=500, epochs=60, log=lambda *a: None)
    if rank == 0:
        out = {"metric": "searchlight ridge grid searches/sec, learned proposal with grid fallback",
               "value": res["learned"]["searchlights_per_s"], "unit": UNIT, "n_gpus": 1, "steps": 1, "warmup": 1,
               "ms_per_step": res["learned"]["ms"], "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f64 (proposal bf16)", "data": "synthetic",
               "config": {"workload": "ridge_grid_learned", "nv": nv, "nt": 500, "fit_rows": 400, "eval_rows": 100,
                          "searchlight_subset": "every 4th", "sizes": "50-500",
                          "noise": "AR(1) rho 0.5, amplitude 0.2 to 6 over the sphere",
                          "train_seeds": [1, 2, 3, 4], "heldout_seed": 5, "min_prob": 0.6},
               "study": res}
        print(json.dumps(out))


# ---------------------------------------------------------------------------------------------
# rank-deficient template pair: about 10% of searchlights hold a duplicated vertex column
# ---------------------------------------------------------------------------------------------

def range_part(T, A, rel=1e-9):
    """T restricted to the row space of A, the part of the polar factor that A determines."""
    _, sv, Vt = np.linalg.svd(A)
    Vp = Vt[sv > sv[0] * rel].T
    return T @ Vp @ Vp.T


def rankdef_errors(w, singular, sample, Ts, fp64_flags):
    """Per-T relative Frobenius error vs the float64 oracle, split into singular searchlights (T
    compared on the row space of A) and regular ones, and by whether the searchlight went to FP64."""
    from oracle import ha_oracle as O
    groups = {"singular": [], "regular": [], "fp64": [], "fp32": []}
    for j, q in enumerate(sample):
        sl = w.sls.indices[w.sls.offsets[q]:w.sls.offsets[q + 1]]
        Xs, Ys = w.X[:, sl], w.Y[:, sl]
        Tref = O.procrustes(Xs, Ys, True, False)
        if singular[q]:
            A = Xs.T @ Ys
            a, b = range_part(Ts[j], A), range_part(Tref, A)
        else:
            a, b = Ts[j], Tref
        e = float(np.linalg.norm(a - b) / np.linalg.norm(b))
        groups["singular" if singular[q] else "regular"].append(e)
        groups["fp64" if fp64_flags[j] else "fp32"].append(e)
    return {k: ({"T_relfrob_max": float(np.max(v)), "T_relfrob_median": float(np.median(v)), "count": len(v)}
                if v else {"count": 0}) for k, v in groups.items()}


# ---------------------------------------------------------------------------------------------
# one hemisphere sharded over the ranks (strong scaling)
# ---------------------------------------------------------------------------------------------

def run_shard(args):
    """The template pair's hemisphere (seed 0 on every rank) split over the N ranks: contiguous
    searchlight ranges balanced by n^3, one all-to-all of partial CSC values per step to the
    column owners. value = searchlights of the hemisphere x steps / max over ranks of the device
    time (solve + exchange)."""
    import torch
    import torch.distributed as dist
    from hyperalignment_b200 import _lib as L
    from hyperalignment_b200.plan import Plan
    from hyperalignment_b200.shard import ShardedSearchlights

    ws, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    lib = L.lib()
    L.check(lib.ha_b200_init(), "ha_b200_init")
    w = workload(0, args.nv, args.nt)
    s = w.sls
    dev = torch.device("cuda", local)
    sh = ShardedSearchlights(w.nt, w.nv, s.indices, s.offsets, s.dists, s.radius)
    hX = torch.from_numpy(np.asfortranarray(w.X).ravel(order="F")).pin_memory()
    hY = torch.from_numpy(np.asfortranarray(w.Y).ravel(order="F")).pin_memory()
    dX, dY = hX.to(dev), hY.to(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step():
        return sh.procrustes(dX, dY, True, True, L.SOLVER_MIXED)

    for _ in range(args.warmup):
        owned = step()
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.5)
    n0 = lib.ha_b200_launch_count()
    torch.cuda.synchronize()
    evs = []
    for _ in range(args.steps):
        flush.zero_()
        a, m, b = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        a.record(stream)
        sh.partial.zero_()
        if sh.plan is not None:
            sh.plan.procrustes_device(dX.data_ptr(), dY.data_ptr(), sh.partial.data_ptr(), True, True,
                                      L.SOLVER_MIXED, L.OUT_CSC, stream.cuda_stream)
        m.record(stream)
        owned = sh.exchange.combine(sh.partial)
        b.record(stream)
        evs.append((a, m, b))
    torch.cuda.synchronize()
    launches = lib.ha_b200_launch_count() - n0
    clocks = sampler.stop()
    K = args.steps
    job_ms = max_over_ranks(sum(a.elapsed_time(b) for a, _, b in evs), ws, dev)
    solve_ms = max_over_ranks(sum(a.elapsed_time(m) for a, m, _ in evs), ws, dev)
    exch_ms = max_over_ranks(sum(m.elapsed_time(b) for _, m, b in evs), ws, dev)
    value = s.count * K / (job_ms / 1e3)

    # end to end: every step copies X and Y from pinned host memory and the owned values back
    hout = torch.empty(owned.numel(), dtype=torch.float64).pin_memory()
    for _ in range(args.warmup):
        dX.copy_(hX, non_blocking=True)
        dY.copy_(hY, non_blocking=True)
        hout.copy_(step(), non_blocking=True)
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    ee = []
    for _ in range(K):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        dX.copy_(hX, non_blocking=True)
        dY.copy_(hY, non_blocking=True)
        hout.copy_(step(), non_blocking=True)
        b.record(stream)
        ee.append((a, b))
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in ee), ws, dev)

    # the sharded result against one plan of the whole hemisphere on rank 0
    full = sh.exchange.assemble(owned, dst=0)
    check = None
    if rank == 0:
        one = Plan.from_workload(w)
        ref = torch.zeros(one.nnz, dtype=torch.float64, device=dev)
        one.procrustes_device(dX.data_ptr(), dY.data_ptr(), ref.data_ptr(), True, True, L.SOLVER_MIXED, L.OUT_CSC,
                              stream.cuda_stream)
        torch.cuda.synchronize()
        indptr, rows = one.pattern()
        refv = ref.cpu().numpy()
        same = bool(np.array_equal(full[0], indptr) and np.array_equal(full[1], rows))
        check = {"pattern_identical": same,
                 "values_relfrob": float(np.linalg.norm(full[2] - refv) / np.linalg.norm(refv)) if same else None}
        # the evaluation step on the same data: A = X @ W and its per-vertex correlation with Y
        r = torch.empty(w.nv, dtype=torch.float64, device=dev)
        A = torch.empty(w.nt * w.nv, dtype=torch.float64, device=dev)
        for _ in range(2):
            one.aligned_correlation_device(dX.data_ptr(), dY.data_ptr(), ref.data_ptr(), r.data_ptr(), A.data_ptr(),
                                           stream=stream.cuda_stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(K):
            one.aligned_correlation_device(dX.data_ptr(), dY.data_ptr(), ref.data_ptr(), r.data_ptr(), A.data_ptr(),
                                           stream=stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ev_ms = e0.elapsed_time(e1) / K
        evaluation = {"kernel": "k_aligned_corr", "ms": ev_ms, "nnz": int(one.nnz), "mean_r": float(r.mean()),
                      "gflops": 2.0 * one.nnz * w.nt / (ev_ms / 1e3) / 1e9,
                      "hbm_gbs_min_bytes": 4.0 * w.nt * w.nv * 8 / (ev_ms / 1e3) / 1e9,
                      "note": "X in L2 between steps (no flush); min bytes = X, Y once, A written and read"}
        check["evaluation"] = evaluation
        one.close()
    if rank == 0:
        lo, hi = sh.col_range
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": K, "warmup": args.warmup,
            "ms_per_step": job_ms / K, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": config_dict(w, {"workload": "hemisphere_template_pair_sharded",
                                      "parallelism": f"one hemisphere over {ws} GPU(s): contiguous searchlight "
                                                     "ranges balanced by n^3, column owners, one all-to-all of "
                                                     "partial CSC values per step"}),
            "solve_ms_per_step": solve_ms / K, "exchange_ms_per_step": exch_ms / K,
            "searchlights_rank0": int(sh.bounds[1] - sh.bounds[0]), "columns_rank0": [int(lo), int(hi)],
            "vs_one_plan": check,
            "e2e": {"value": s.count * K / (e2e_ms / 1e3), "unit": UNIT,
                    "h2d_bytes_per_step": int(2 * w.nt * w.nv * 8), "d2h_bytes_per_step": int(owned.numel() * 8),
                    "path": "ShardedSearchlights.procrustes with X, Y copied from pinned host memory and the "
                            "owned CSC values copied back every step (rank 0's bytes)"},
            "roofline": None, "cpu_baseline": None,
            "gpu_launches": int(launches), "clocks": clocks,
        }
        print(json.dumps(out))
    sh.close()
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()


# ---------------------------------------------------------------------------------------------
# the shapes of the reference's published run (StudyForrest: nt 1818, ~9,675 searchlights of 90-170)
# ---------------------------------------------------------------------------------------------

# The reference's published per-hemisphere timings of this run (the reference project's README.md:223-241), as
# searchlights/s = 9,675 / seconds per hemisphere, for context: other hardware, the real data set.
PUBLISHED_FORREST = {"c_cuda_fp32_rtx4090": 459, "c_cpu_fp32_96_threads_tr7995wx": 15100,
                     "c_cpu_fp64_96_threads_tr7995wx": 8880, "c_cpu_fp32_10_threads_m4pro": 7740}


def run_forrest(args):
    """Dense searchlight Procrustes (reflection allowed, no scaling, distance weights) on synthetic
    inputs with the shapes of the reference's published run: device-resident steps (value) and the
    C-ABI dense entry from host buffers into a host nv x nv matrix (e2e, the published runs' form)."""
    import torch
    from hyperalignment_b200 import _lib as L
    from hyperalignment_b200 import workloads as W
    from hyperalignment_b200.plan import Plan
    torch.cuda.set_device(0)
    lib = L.lib()
    L.check(lib.ha_b200_init(), "ha_b200_init")
    w = W.forrest_shaped(0)
    s = w.sls
    dev = torch.device("cuda", 0)
    plan = Plan.from_workload(w)
    dX = torch.from_numpy(np.asfortranarray(w.X).ravel(order="F")).to(dev)
    dY = torch.from_numpy(np.asfortranarray(w.Y).ravel(order="F")).to(dev)
    vals = torch.zeros(plan.nnz, dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step():
        plan.procrustes_device(dX.data_ptr(), dY.data_ptr(), vals.data_ptr(), True, False, L.SOLVER_MIXED,
                               L.OUT_CSR, stream.cuda_stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    sampler = ClockSampler(0)
    sampler.start()
    n0 = lib.ha_b200_launch_count()
    evs = []
    for _ in range(args.steps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        step()
        b.record(stream)
        evs.append((a, b))
    torch.cuda.synchronize()
    launches = lib.ha_b200_launch_count() - n0
    clocks = sampler.stop()
    K = args.steps
    ms = sum(a.elapsed_time(b) for a, b in evs)
    stats = plan.stats()

    e2e = None
    if not args.no_e2e:
        Xf, Yf = np.asfortranarray(w.X), np.asfortranarray(w.Y)
        T_out = np.zeros((w.nv, w.nv))
        argsv = (Xf.ctypes.data_as(L.c_double_p), Yf.ctypes.data_as(L.c_double_p), w.nt, w.nv, L.iptr(s.indices),
                 L.iptr(s.offsets), L.dptr(s.dists), s.count, s.radius, T_out.ctypes.data_as(L.c_double_p), True,
                 False, L.BACKEND_B200, True)
        lib.ha_set_num_threads(os.cpu_count() or 1)
        L.check(lib.ha_searchlight_procrustes_dense(*argsv), "dense")
        ts = []
        for _ in range(max(1, K - 1)):
            t0 = time.perf_counter()
            L.check(lib.ha_searchlight_procrustes_dense(*argsv), "dense")
            ts.append(time.perf_counter() - t0)
        e2e = {"value": s.count * len(ts) / sum(ts), "unit": UNIT, "h2d_bytes_per_step": int(2 * w.nt * w.nv * 8),
               "d2h_bytes_per_step": int(plan.nnz * 8),
               "path": "ha_searchlight_procrustes_dense(backend=4), host float64 in, host dense nv x nv out (+=); "
                       "wall clock per call"}

    from oracle import ha_oracle as O
    rng = np.random.default_rng(5)
    sample = np.sort(rng.choice(s.count, size=12, replace=False))
    sub = s.subset(sample)
    splan = Plan(w.nt, w.nv, sub.indices, sub.offsets, sub.dists, sub.radius)
    svals = torch.zeros(splan.nnz, dtype=torch.float64, device=dev)
    splan.procrustes_device(dX.data_ptr(), dY.data_ptr(), svals.data_ptr(), True, False, L.SOLVER_MIXED, L.OUT_CSR,
                            stream.cuda_stream)
    torch.cuda.synchronize()
    Ts = splan.local_transforms(0, sub.count)
    err = []
    for j, q in enumerate(sample):
        sl = s.indices[s.offsets[q]:s.offsets[q + 1]]
        Tref = O.procrustes(w.X[:, sl], w.Y[:, sl], True, False)
        err.append(np.linalg.norm(Ts[j] - Tref) / np.linalg.norm(Tref))
    splan.close()
    sizes = s.sizes
    out = {
        "metric": METRIC, "value": s.count * K / (ms / 1e3), "unit": UNIT, "n_gpus": 1, "steps": K,
        "warmup": args.warmup, "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": "forrest_shaped", "nv": w.nv, "nt": w.nt, "searchlights": s.count,
                   "sl_size_min": int(sizes.min()), "sl_size_max": int(sizes.max()),
                   "sl_size_mean": round(float(sizes.mean()), 2), "reflection": True, "scaling": False,
                   "weights": "linear distance", "l2": "flushed between steps (256 MiB write)"},
        "e2e": e2e, "error_vs_fp64": {"T_relfrob_max": float(max(err)), "T_relfrob_median": float(np.median(err)),
                                      "sample": len(err)},
        "solver_stats": stats, "gpu_launches": int(launches), "clocks": clocks,
        "published_reference_searchlights_per_s": PUBLISHED_FORREST,
    }
    print(json.dumps(out))
    plan.close()


def run_pca(args):
    """Searchlight PCA template (the Python package's searchlight_template(tpl_kind="pca"),
    src/hyperalignment/searchlight.py:215-236) on the hemisphere of the template workload: 10242
    searchlights of 100-300 vertices, 10 subjects, nt 400, through the C entry from host buffers
    (every step uploads the subjects and downloads the template).  The float64 CPU oracle (exact SVD
    per searchlight) is timed on a sample of searchlights, and the GPU template of the same sample
    is checked against it."""
    import torch
    from threadpoolctl import threadpool_info
    from hyperalignment_b200 import _lib as L
    from hyperalignment_b200 import hyperalignment_c as H
    from hyperalignment_b200 import workloads as W
    from oracle import ha_oracle as O
    torch.cuda.set_device(0)
    lib = L.lib()
    L.check(lib.ha_b200_init(), "ha_b200_init")
    _, sls, subj = W.hemisphere_subjects(seed=0, nv=args.nv, nt=args.nt, n_subj=10, size_lo=100, size_hi=300)
    ns, nt, nv = len(subj), args.nt, args.nv
    stack = np.empty((ns, nv, nt))
    for j, D in enumerate(subj):
        stack[j] = D.T
    out = np.empty((nv, nt))
    argv = (L.dptr(stack), ns, nt, nv, L.iptr(sls.indices), L.iptr(sls.offsets), L.dptr(sls.dists), sls.count,
            float(sls.radius), L.dptr(out))

    def step():
        L.check(lib.ha_searchlight_pca_template_b200(*argv), "ha_searchlight_pca_template_b200")

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    sampler = ClockSampler(0)
    sampler.start()
    time.sleep(0.5)
    n0 = lib.ha_b200_launch_count()
    evs, walls = [], []
    for _ in range(args.steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        a.record(stream)
        step()
        b.record(stream)
        torch.cuda.synchronize()
        walls.append(time.perf_counter() - t0)
        evs.append((a, b))
    launches = lib.ha_b200_launch_count() - n0
    clocks = sampler.stop()
    K = args.steps
    ms = sum(a.elapsed_time(b) for a, b in evs)
    # kernel time of one traced step (CUDA events around every launch)
    lib.ha_b200_kernel_times(None, None)
    lib.ha_b200_set_kernel_timing(True)
    step()
    lib.ha_b200_set_kernel_timing(False)
    kms = np.zeros(len(L.KERNEL_KINDS))
    kcnt = np.zeros(len(L.KERNEL_KINDS), dtype=np.int64)
    lib.ha_b200_kernel_times(kms.ctypes.data_as(L.c_double_p), kcnt.ctypes.data_as(L.c_int64_p))
    # CPU oracle on a growing sample of searchlights, and the GPU template of the same sample
    rng = np.random.default_rng(3)
    order = rng.permutation(sls.count)
    take, cpu_s = 4, 0.0
    while True:
        sample = np.sort(order[:take])
        sub = sls.subset(sample)
        t0 = time.perf_counter()
        ref = O.searchlight_pca_template(subj, sub.indices, sub.offsets, sub.dists, sub.radius)
        cpu_s = time.perf_counter() - t0
        if cpu_s >= args.cpu_seconds or take >= sls.count:
            break
        take = min(sls.count, max(take * 2, int(take * args.cpu_seconds / max(cpu_s, 1e-3) * 1.1)))
    got = H.searchlight_pca_template(subj, [sub.indices[sub.offsets[q]:sub.offsets[q + 1]] for q in range(sub.count)],
                                     [sub.dists[sub.offsets[q]:sub.offsets[q + 1]] for q in range(sub.count)],
                                     sub.radius)
    err = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
    blas = max((i.get("num_threads", 1) for i in threadpool_info()), default=1)
    sizes = sls.sizes
    value = sls.count * K / (ms / 1e3)
    res = {
        "metric": "searchlight PCA template: searchlights/s", "value": value, "unit": "searchlights/s", "n_gpus": 1,
        "steps": K, "warmup": args.warmup, "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "hemisphere_pca_template", "nv": nv, "nt": nt, "subjects": ns,
                   "searchlights": sls.count, "sl_size_min": int(sizes.min()), "sl_size_max": int(sizes.max()),
                   "sl_size_mean": round(float(sizes.mean()), 2), "gram_order": int(min(nt, ns * sizes.min())),
                   "weights": "linear distance",
                   "l2": "inputs (328 MB of subjects) larger than L2, uploaded every step"},
        "timing": "CUDA events on the default stream around the C entry (host float64 in, host template out)",
        "e2e": {"value": sls.count * K / sum(walls), "unit": "searchlights/s",
                "h2d_bytes_per_step": int(stack.nbytes), "d2h_bytes_per_step": int(out.nbytes),
                "path": "ha_searchlight_pca_template_b200, wall clock per call"},
        "kernel_ms_per_step": {L.KERNEL_KINDS[i]: round(float(kms[i]), 3) for i in range(len(L.KERNEL_KINDS))
                               if kcnt[i] > 0},
        "kernel_kinds": "pca: k_pca_gram, k_pca_tmpl, k_pca_contrib, k_pca_reduce; ridge: k_pchol; jacobi64: "
                        "k_jacobi<double> (eigenvector mode on the Gram factors, then the polar); formT64: "
                        "k_form_t_global<double>",
        "error_vs_oracle": {"template_relfrob": err, "sample": int(sub.count)},
        "cpu_baseline": {"value": sub.count / cpu_s, "unit": "searchlights/s", "cores": int(blas), "kind": "port",
                         "sample": f"{sub.count} random searchlights, oracle exact-SVD template (numpy LAPACK, "
                                   f"{blas} BLAS threads), {cpu_s:.1f} s"},
        "gpu_launches": int(launches), "clocks": clocks,
    }
    print(json.dumps(res))


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "grid":
        run_grid(args)
    elif args.workload == "learned":
        run_learned(args)
    elif args.workload == "shard":
        run_shard(args)
    elif args.workload == "forrest":
        run_forrest(args)
    elif args.workload == "refgpu":
        run_refgpu(args)
    elif args.workload == "pca":
        run_pca(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
