#!/usr/bin/env python
"""Benchmark of the B200 coordinate-descent engine.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: Poisson regression with offset, N=1,000,000 rows x P=100,000
covariates (rank-Zipf(1.1) column sizes capped at 50,000, ~2e7 nonzeros, 80 %
indicator / 20 % sparse LogNormal columns), offset log(t), intercept, Normal
prior variance 1, FP64, the reference's default convergence (gradient, 1e-6).
Seeded synthetic data of that shape (no public dataset exists for it).

A step is one converged findMode from a cold start (beta = 0, offset 1): the
whole coordinate-descent hot path over one input.  `value` is coordinate
updates per second with the inputs resident in HBM (device-timed with CUDA
events on the engine's stream, max over ranks, L2 flushed between steps);
`e2e` is the same metric through the one-call C-ABI entry point
(ccdb_fit_model) from pinned host buffers, uploads and the copy of beta back
inside the timed span.  With --gpus N each rank fits its own replica (weak
scaling; a single fit does not shard).

--impl reference times the reference Cyclops engine compiled from source (or
the plain-C restatement where it is absent) on the host cores, one sweep of
the same workload per step.
"""
from __future__ import annotations

import argparse
import collections
import json
import os
import subprocess
import sys
import tempfile
import time
from typing import Optional

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from ccd_b200 import synthetic  # noqa: E402
from ccd_b200.data import DENSE, GRADIENT, INDICATOR, INTERCEPT, SPARSE  # noqa: E402

METRIC = "coord-updates/s"
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--small", action="store_true", help="a 10x smaller problem (quick checks)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="headline only: skip the other configurations' measurements nested in the line")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the converged oracle fit that the headline line's parity fields compare with")
    ap.add_argument("--max-sweeps", type=int, default=1000,
                    help="cap on sweeps per findMode (profiling captures of one short launch)")
    ap.add_argument("--serve-requests", type=int, default=200,
                    help="serve: requests in the replayed stream")
    ap.add_argument("--serve-slots", type=int, default=8, help="serve: concurrent fits")
    ap.add_argument("--serve-fast-ctas", type=int, default=1, help="serve: CTAs of a fast slot's fit")
    ap.add_argument("--serve-detail", default=None, metavar="PATH",
                    help="serve: write per-request wait/service times of the last replay, and each "
                         "request's time alone, as JSON lines to PATH")
    ap.add_argument("--serve-slot-ctas", type=int, default=0,
                    help="serve: at most this many CTAs for a general slot's fit (0: an even share)")
    ap.add_argument("--serve-fast-slots", type=int, default=4,
                    help="serve: extra slots that take only small requests (at most 200,000 entries)")
    ap.add_argument("--workload", choices=["poisson_offset", "logistic_l1", "cv_grid", "cox_breslow", "serve",
                                           "kkt_l1", "mm_clr", "fisher_l1"],
                    default="poisson_offset",
                    help="poisson_offset: plain fits (default); cv_grid: 10 folds x 20 Laplace "
                         "variances = 200 logistic fits over one shared 5e5 x 2e4 matrix; "
                         "kkt_l1 / mm_clr / fisher_l1: the mode-finding variants and the Fisher "
                         "information (see variant_problem)")
    ap.add_argument("--plain-sample", type=int, default=3,
                    help="cv_grid: instances also fitted one at a time by the plain solver")
    ap.add_argument("--precision", choices=["mixed", "fp64"], default="mixed",
                    help="cv_grid: the mixed-precision lockstep engine (default) or the FP64 one")
    ap.add_argument("--cluster", type=int, default=0,
                    help="cv_grid, mixed, with --group: CTAs per group (0: the engine's choice)")
    ap.add_argument("--group", type=int, default=0,
                    help="cv_grid, mixed: instances per lockstep group (0: the engine's choice)")
    ap.add_argument("--cv-columns", type=int, default=20_000,
                    help="cv_grid: covariate columns (fewer for short profiling captures)")
    ap.add_argument("--fp64-check", type=int, default=4,
                    help="cv_grid, mixed: instances also fitted by the FP64 engine to report the error")
    ap.add_argument("--strategy", choices=["auto", "levels", "speculative", "grid_levels", "resident"], default="auto",
                    help="sweep strategy of the independent-row engine (CCDB_SWEEP_*)")
    ap.add_argument("--trace", default=None,
                    help="write a per-level timestamp trace of the last timed findMode's first "
                         "sweep to this file (summarise with python -m ccd_b200.trace)")
    return ap.parse_args()


WORKLOAD = "poisson_offset"


def workload(rank: int, small: bool):
    if WORKLOAD == "cox_breslow":
        if small:
            return synthetic.cox_breslow(seed=3 + rank, K=100_000, n_strata=100, P=5_000)
        return synthetic.cox_breslow(seed=3 + rank)
    if small:
        d = synthetic.poisson_offset(seed=2 + rank, K=100_000, P=10_000, total_nnz=2e6, cap=5_000)
    else:
        d = synthetic.poisson_offset(seed=2 + rank)
    return d


def config_of(d, small: bool) -> dict:
    """The workload, the same on both arms; what one timed step covers is the
    line's own `step` key (a converged fit here, a sweep on the reference arm:
    the metric is per coordinate update, and the reference's cost per sweep is
    flat over a fit)."""
    if WORKLOAD == "cox_breslow":
        return {
            "workload": "cox_breslow" + ("_small" if small else ""), "model": "cox (Breslow ties)",
            "rows": d.K, "columns": d.J, "nnz": d.nnz, "strata": int(d.stratum.max()) + 1,
            "prior": "laplace(0.05)", "convergence": "gradient, tol 1e-6", "precision": "fp64",
            "start": "cold (beta = 0)",
        }
    return {
        "workload": "poisson_offset" + ("_small" if small else ""),
        "model": "poisson",
        "rows": d.K, "columns": d.J, "nnz": d.nnz,
        "prior": "normal(1.0), none on offset/intercept",
        "convergence": "gradient, tol 1e-6",
        "precision": "fp64",
        "start": "cold (beta = 0, offset 1)",
    }


def column_slice(d, n_cols: int):
    """The first n_cols columns of a problem (same rows, strata, times)."""
    from ccd_b200.data import CyclopsData
    n = min(n_cols, d.J)
    cs = d.col_start[:n + 1].copy()
    vs = d.val_start[:n + 1].copy()
    return CyclopsData(d.model_type, d.y, cs, d.rows[:cs[-1]], vs, d.vals[:vs[-1]], d.fmt[:n],
                       d.prior_type[:n], d.prior_var[:n], time=d.time, stratum=d.stratum,
                       offset_col0=d.offset_col0)


def cold_beta(d) -> np.ndarray:
    b = np.zeros(d.J)
    if d.offset_col0:
        b[0] = 1.0
    return b


def active_columns(d) -> int:
    return d.J - (1 if d.offset_col0 else 0)


def sweep_bytes(d) -> float:
    """Algorithmic bytes of one sweep (FP64, unweighted, every delta nonzero):
    per entry the column index (4 B, SPARSE/INDICATOR) and value (8 B, SPARSE/
    DENSE) read for the gradient and again for the update, plus one 8-byte row
    state word read for the gradient and read+written by the update."""
    total = 0.0
    lo = 1 if d.offset_col0 else 0
    cnt = np.diff(d.col_start)
    for f, idx_b, val_b in ((INDICATOR, 4, 0), (SPARSE, 4, 8), (DENSE, 0, 8), (INTERCEPT, 0, 0)):
        sel = d.fmt[lo:] == f
        if f in (DENSE, INTERCEPT):
            e = float(sel.sum()) * d.K
        else:
            e = float(cnt[lo:][sel].sum())
        total += e * (idx_b + val_b) * 2 + e * 8 * 3
    return total


def cox_groups(d) -> int:
    """Risk-set tie groups of an unweighted Breslow Cox problem (rows sorted by
    stratum, -time, y): a row starts a new group unless the previous row of its
    stratum is an event at the same time with the same outcome
    (setPidForAccumulation, ModelSpecifics.hpp:1809-1868)."""
    s, t, y = d.stratum, d.time, d.y
    same = (s[1:] == s[:-1]) & (y[:-1] == 1.0) & (t[1:] == t[:-1]) & (y[1:] == y[:-1])
    return int(1 + np.count_nonzero(~same))


def cox_bytes(d, sweeps: int, nonzero_steps: int) -> float:
    """Algorithmic bytes of the Cox fits' sweeps on this engine: every
    coordinate's O(nnz) gradient reads, per entry, the row id (4 B), {xBeta, e}
    (16 B), the row's group and stratum (8 B) and the group's suffix sums S1, S2
    (16 B); every nonzero step reads and writes its column's rows (4 + 16 + 16
    B), records and applies each row's change to its group (16 B), and rebuilds
    the accumulated denominators and suffix sums over every group (denominator
    read, D written; D and events read, S1 and S2 written: 48 B per group).
    The reference's own walk over every group for every coordinate
    (ModelSpecifics.hpp:904-964) is not counted: this engine does not do it."""
    lo = 1 if d.offset_col0 else 0
    cnt = np.diff(d.col_start)[lo:].astype(np.float64)
    grad = float(cnt.sum()) * 44.0
    avg = float(cnt.mean()) if len(cnt) else 0.0
    return sweeps * grad + nonzero_steps * (avg * 52.0 + 48.0 * cox_groups(d))


def objective_bytes(d) -> float:
    """One convergence check: y and xBeta of every row."""
    return d.K * 16.0


def read_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as fh:
            v = json.load(fh)
        return float(v["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def read_traffic(workload_name: str):
    """Per-launch DRAM bytes of the sweep kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", f"sweep_{workload_name}.md")
    try:
        with open(p) as fh:
            for line in fh:
                if line.strip().startswith("traffic_bytes_per_sweep:"):
                    return float(line.split(":", 1)[1].split()[0])
    except (OSError, ValueError, IndexError):
        pass  # not captured yet: traffic is reported as null
    return None


class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as fh:
            for line in fh:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax = float(parts[2])
                except ValueError:
                    continue
                for n, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def allreduce(vals, op, world):
    """All-reduce a few floats over the ranks (NCCL on GPUs, gloo on CPU)."""
    if world == 1:
        return vals
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor(vals, dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return t.tolist()


def cv_shard(n: int, world: int, rank: int) -> np.ndarray:
    """Instances of a cross-validation grid fitted by `rank`: round robin over the
    grid, so that every rank gets a share of the weak priors (the longest fits)."""
    return np.arange(rank, n, world)


def cpu_reference_sample(d, target_s: float = 15.0):
    """The reference CPU engine on a bounded sample of the same workload: the
    first n sweeps of the cold-start fit, single thread."""
    from oracle import checker
    eng_cls = checker.best_engine()
    kind = "reference" if eng_cls is checker.ReferenceEngine else "port"
    if WORKLOAD == "cox_breslow":
        # O(#groups) per coordinate in the reference: time the first sweep over a
        # 2,000-column slice of the same data (rows, strata, times unchanged)
        ds = column_slice(d, 2000)
        eng = eng_cls(ds)
        t0 = time.perf_counter()
        eng.fit(GRADIENT, 1e-6, max_iter=1)
        t1 = time.perf_counter() - t0
        eng.close()
        return {"value": ds.J / t1, "unit": METRIC, "cores": 1, "kind": kind,
                "sample": f"first sweep over the first {ds.J} columns of the same rows/strata "
                          f"({ds.J} coordinate updates, {t1:.1f} s), single thread"}
    eng = eng_cls(d)
    t0 = time.perf_counter()
    eng.fit(GRADIENT, 1e-6, max_iter=1)
    t1 = time.perf_counter() - t0
    n = int(max(1, min(20, round(target_s / max(t1, 1e-3)))))
    if n > 1:
        eng.set_beta(cold_beta(d))
        t0 = time.perf_counter()
        eng.fit(GRADIENT, 1e-6, max_iter=n)
        tn = time.perf_counter() - t0
    else:
        tn = t1
    eng.close()
    rate = n * active_columns(d) / tn
    return {"value": rate, "unit": METRIC, "cores": 1, "kind": kind,
            "sample": f"first {n} sweep(s) of the cold-start fit ({n * active_columns(d)} coordinate "
                      f"updates, {tn:.1f} s), single thread (the reference inner loop is serial)"}


class ConvergedReference:
    """The same problem fitted to convergence on the host cores, beside the GPU
    steps (threads; the GPU's timed region holds only device work): the oracle
    restatement, bit-identical with the reference engine on every pinned case,
    for the coefficients, log-likelihood, return flag and the cycles of each
    findMode attempt; and the compiled reference engine, where present, for its
    time to converge.  Single thread each, as the reference's inner loop is
    serial."""

    def __init__(self, d, conv: int, tol: float, fit_kw: Optional[dict] = None):
        import threading
        self.d, self.conv, self.tol, self.kw = d, conv, tol, fit_kw or {}
        self.port = None
        self.ref_seconds = None
        self.ref_kind = None
        self.error = None
        self.threads = [threading.Thread(target=self._port, daemon=True),
                        threading.Thread(target=self._reference, daemon=True)]
        for t in self.threads:
            t.start()

    def _port(self):
        from oracle import checker
        try:
            e = checker.RestatementEngine(self.d)
            t0 = time.perf_counter()
            r = e.fit(self.conv, self.tol, **self.kw)
            r["seconds"] = time.perf_counter() - t0
            r["attempt_sweeps"] = e.fit_attempts()
            e.close()
            self.port = r
        except Exception as ex:  # reported in the line, never fatal to the bench
            self.error = f"restatement: {ex}"

    def _reference(self):
        from oracle import checker
        if not checker.reference_available():
            return
        try:
            e = checker.ReferenceEngine(self.d)
            t0 = time.perf_counter()
            e.fit(self.conv, self.tol, **self.kw)
            self.ref_seconds = time.perf_counter() - t0
            self.ref_kind = "reference"
            e.close()
        except Exception as ex:
            self.error = f"reference: {ex}"

    def result(self, beta, loglik, flag, iterations, attempt_sweeps) -> dict:
        """Errors of a GPU fit against the converged restatement."""
        for t in self.threads:
            t.join()
        if self.port is None:
            return {"error": self.error}
        w = self.port
        scale = max(float(np.max(np.abs(w["beta"]))), 1e-8)
        return {
            "oracle": "FP64 restatement of the reference (bit-identical with it on every pinned case)",
            "max_rel_dbeta": float(np.max(np.abs(np.asarray(beta) - w["beta"]))) / scale,
            "rel_dll": abs(loglik - w["loglik"]) / max(1.0, abs(w["loglik"])),
            "return_flag": {"gpu": int(flag), "oracle": int(w["flag"])},
            "iterations": {"gpu": int(iterations), "oracle": int(w["iterations"])},
            "attempt_sweeps": {"gpu": [int(x) for x in attempt_sweeps], "oracle": w["attempt_sweeps"]},
            "oracle_seconds": w["seconds"],
            "within_tolerance": bool(float(np.max(np.abs(np.asarray(beta) - w["beta"]))) <= 1e-6 * scale
                                     and abs(loglik - w["loglik"]) <= 1e-9 * max(1.0, abs(w["loglik"]))
                                     and int(flag) == int(w["flag"])),
        }


def run_reference(args, world, rank):
    if rank != 0:
        return
    from oracle import checker
    d = workload(0, args.small)
    eng_cls = checker.best_engine()
    kind = "reference" if eng_cls is checker.ReferenceEngine else "port"
    eng = eng_cls(d)
    # one whole fit to convergence first (time to converge, the ILLCONDITIONED retry
    # included), then the per-step samples: one sweep each
    eng.set_beta(cold_beta(d))
    t0 = time.perf_counter()
    conv_fit = eng.fit(GRADIENT, 1e-6)
    conv_t = time.perf_counter() - t0
    times = []
    for i in range(args.warmup + args.steps):
        eng.set_beta(cold_beta(d))
        t0 = time.perf_counter()
        eng.fit(GRADIENT, 1e-6, max_iter=1)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            times.append(dt)
    eng.close()
    total = float(np.sum(times))
    v = args.steps * active_columns(d) / total
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": METRIC, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded PCG64, workload shapes of the benchmark config)",
        "config": config_of(d, args.small),
        "step": "one sweep of the cold-start fit (a bounded sample; the cost per sweep is flat over a fit)",
        "time_to_converge_s": conv_t,
        "converged_fit": {"iterations": int(conv_fit["iterations"]), "return_flag": int(conv_fit["flag"]),
                          "log_likelihood": float(conv_fit["loglik"])},
        "cpu_baseline": {"value": v, "unit": METRIC, "cores": 1, "kind": kind,
                         "sample": "one sweep of the cold-start fit per step, single thread; "
                                   "time_to_converge_s is one whole fit, timed once before the steps"},
        "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, world, rank, local, collect=False):
    import torch
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from ccd_b200 import native
    import torch.distributed as tdist

    d = workload(rank, args.small)
    ctx = native.Context(local)
    m = native.Matrix(ctx, d)
    f = native.Fit(ctx, m, d)
    margs = native.ModeFindingArguments(convergence_type=GRADIENT, tolerance=1e-6,
                                        max_iterations=args.max_sweeps, strategy=STRATEGIES[args.strategy])
    cold = cold_beta(d)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=f"cuda:{local}")

    parity = (ConvergedReference(d, GRADIENT, 1e-6)
              if rank == 0 and not args.no_parity and WORKLOAD == "poisson_offset" else None)
    for _ in range(args.warmup):
        f.set_beta(cold)
        f.find_mode(margs)

    clocks = Clocks(local)
    if world > 1:
        tdist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    dev_t, ker_t, updates, launches, sweeps, lat = 0.0, 0.0, 0, 0, 0, []
    attempts = nonzero = 0
    for i in range(args.steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        f.set_beta(cold)
        if args.trace and i == args.steps - 1:
            os.environ["CCDB_TRACE_FILE"] = args.trace
        r = f.find_mode(margs)
        os.environ.pop("CCDB_TRACE_FILE", None)
        dev_t += r.device_seconds
        ker_t += r.kernel_seconds
        updates += r.coordinate_updates
        launches += r.kernel_launches
        sweeps += r.sweeps_total
        attempts += r.attempts
        nonzero += max(0, r.nonzero_steps)
        lat.append(r.device_seconds)
    torch.cuda.synchronize()
    if world > 1:
        tdist.barrier()
    clk = clocks.stop()
    last = r

    # end to end through the one-call entry point, inputs in pinned host memory
    def pinned(a):
        t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
        return t.numpy()
    from ccd_b200.data import CyclopsData
    dp = CyclopsData(d.model_type, pinned(d.y), pinned(d.col_start), pinned(d.rows),
                     pinned(d.val_start), pinned(d.vals), pinned(d.fmt), d.prior_type, d.prior_var,
                     time=d.time, stratum=d.stratum, offset_col0=d.offset_col0)
    h2d = sum(a.nbytes for a in (dp.y, dp.col_start, dp.rows, dp.val_start, dp.vals, dp.fmt))
    d2h = d.J * 8
    e2e_t, e2e_updates = 0.0, 0
    e2e_steps = args.steps
    if world > 1:
        tdist.barrier()
    torch.cuda.synchronize()
    for _ in range(e2e_steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        r2 = native.fit_model(ctx, dp, margs)
        e2e_t += r2.device_seconds
        e2e_updates += r2.coordinate_updates
    torch.cuda.synchronize()

    mx = allreduce([dev_t, e2e_t], tdist.ReduceOp.MAX if world > 1 else None, world)
    sm = allreduce([float(updates), float(e2e_updates), float(launches)],
                   tdist.ReduceOp.SUM if world > 1 else None, world)
    dev_max, e2e_max = mx
    tot_updates, tot_e2e, tot_launch = sm

    if rank == 0:
        peak, peak_kind = read_peaks()
        # every sweep that ran counts, the ILLCONDITIONED attempts' included; one
        # sweep-kernel launch per findMode attempt, each with its initial objective
        total_bytes = sweep_bytes(d) * sweeps + objective_bytes(d) * (sweeps + attempts)
        per_launch_bytes = total_bytes / attempts
        achieved = total_bytes / ker_t / 1e9
        wl = config_of(d, args.small)["workload"]
        traffic = read_traffic(wl)  # DRAM bytes of one sweep (ncu), scaled to a launch's sweeps
        if traffic is not None:
            traffic = traffic * sweeps / attempts
        n_levels = native.sweep_levels(d)[1]
        attempt_sweeps = [sweeps // args.steps - r.iterations, r.iterations] if r.attempts == 2 \
            else ([r.iterations] if r.attempts == 1 else [r.sweeps_total])
        line = {
            "metric": METRIC, "value": tot_updates / dev_max, "unit": METRIC, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dev_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded PCG64, workload shapes of the benchmark config)",
            "config": config_of(d, args.small),
            "step": "one converged findMode from a cold start",
            "parallelism": f"replicas x{world}",
            "l2": "flushed between timed steps (512 MiB device write)",
            "fits_per_s": world * args.steps / dev_max,
            "fit_latency_ms": {"p50": 1e3 * float(np.percentile(lat, 50)),
                               "p99": 1e3 * float(np.percentile(lat, 99))},
            "sweeps_per_fit": sweeps / args.steps,
            "findmode_attempts_per_fit": attempts / args.steps,
            "dependency_levels_per_sweep": int(n_levels),
            "level_latency_us": 1e6 * ker_t / (sweeps * n_levels),
            "time_to_converge_s": dev_max / args.steps,
            "return_flag": last.return_flag,
            "e2e": {"value": tot_e2e / e2e_max, "unit": METRIC, "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "nonzero_steps_per_fit": nonzero / args.steps,
            "roofline": ({"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                          "frac": achieved / peak, "peak_source": peak_kind,
                          "algorithmic_bytes_per_launch": per_launch_bytes,
                          "kernel": ("cluster_sweep_kernel<POISSON>" if args.strategy != "grid_levels"
                                     else "indep_sweep_kernel<POISSON>") + " (one launch per findMode attempt)",
                          "bytes": "per-coordinate algorithmic bytes (column entries and the row state they gather and update) of every sweep that ran, plus the objective checks",
                          "traffic": traffic} if WORKLOAD == "poisson_offset" else
                         {"bound": "hbm", "achieved": cox_bytes(d, sweeps, nonzero) / ker_t / 1e9, "peak": peak,
                          "unit": "GB/s", "frac": cox_bytes(d, sweeps, nonzero) / ker_t / 1e9 / peak,
                          "peak_source": peak_kind,
                          "algorithmic_bytes_per_launch": cox_bytes(d, sweeps, nonzero) / attempts,
                          "kernel": "group_sweep_kernel<COX> (one launch per findMode attempt)",
                          "bytes": "this engine's O(nnz) gradients plus the O(groups) rebuild per nonzero step "
                                   "(cox_bytes)", "traffic": None}),
            "gpu_launches": int(tot_launch),
            "clocks": clk,
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_reference_sample(d)
        if parity is not None:
            line["parity"] = parity.result(last.beta, last.log_likelihood, last.return_flag, last.iterations,
                                           attempt_sweeps)
            if parity.ref_seconds is not None:
                line["cpu_time_to_converge_s"] = {"value": parity.ref_seconds, "cores": 1,
                                                  "kind": parity.ref_kind}
    if rank == 0 and WORKLOAD == "cox_breslow":
        # the same fit in mixed precision beside FP64, and its error against the FP64 fit
        fm = native.Fit(ctx, m, d, precision=native.PRECISION_MIXED)
        fm.set_beta(cold)
        fm.find_mode(margs)  # warm-up
        fm.set_beta(cold)
        rm = fm.find_mode(margs)
        fm.close()
        scale = max(float(np.max(np.abs(last.beta))), 1e-8)
        line["mixed_precision"] = {
            "ms_per_fit": 1e3 * rm.device_seconds, "iterations": int(rm.iterations),
            "return_flag": int(rm.return_flag), "coordinate_updates_per_s": rm.coordinate_updates / rm.device_seconds,
            "max_rel_dbeta_vs_fp64": float(np.max(np.abs(rm.beta - last.beta))) / scale,
            "rel_dll_vs_fp64": abs(rm.log_likelihood - last.log_likelihood) / max(1.0, abs(last.log_likelihood)),
            "arithmetic": "FP32 exp and per-entry terms (TwoSum), FP64 risk-set sums, reductions, step"}
    f.close()
    m.close()
    ctx.close()
    if rank == 0 and collect:
        return line
    if rank == 0:
        if world == 1 and WORKLOAD == "poisson_offset" and not args.no_extras:
            del flush
            line["workloads"] = run_extras(args, local)
        print(json.dumps(line), flush=True)
    if world > 1:
        tdist.destroy_process_group()


def run_logistic_l1(args, world, rank, local, collect=False):
    """The CPU-runnable configuration: L1 logistic regression, 10,000 rows x
    1,000 indicator covariates at density 0.01 plus an intercept, Laplace
    variance 0.1, FP64, relative log-likelihood change (MITTAL) 1e-6, cold
    start.  A step is one converged fit; the reference engine's converged fit
    of the same problem is timed on the host (single thread, repeated for a
    stable figure) and the oracle's coefficients give the parity fields."""
    import torch
    from ccd_b200 import native
    from ccd_b200.data import MITTAL
    from oracle import checker
    if rank != 0:
        return None
    d = synthetic.logistic_l1(seed=1)
    ctx = native.Context(local)
    m = native.Matrix(ctx, d)
    f = native.Fit(ctx, m, d)
    margs = native.ModeFindingArguments(convergence_type=MITTAL, tolerance=1e-6, max_iterations=args.max_sweeps,
                                        strategy=STRATEGIES[args.strategy])
    cold = cold_beta(d)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=f"cuda:{local}")
    for _ in range(args.warmup):
        f.set_beta(cold)
        f.find_mode(margs)
    clocks = Clocks(local)
    torch.cuda.synchronize()
    clocks.start()
    dev_t = ker_t = 0.0
    sweeps = attempts = launches = 0
    for _ in range(args.steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        f.set_beta(cold)
        r = f.find_mode(margs)
        dev_t += r.device_seconds
        ker_t += r.kernel_seconds
        sweeps += r.sweeps_total
        attempts += r.attempts
        launches += r.kernel_launches
    torch.cuda.synchronize()
    clk = clocks.stop()
    e2e_t = 0.0
    for _ in range(args.steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        e2e_t += native.fit_model(ctx, d, margs).device_seconds
    h2d = sum(a.nbytes for a in (d.y, d.col_start, d.rows, d.val_start, d.vals, d.fmt))
    f.close()
    m.close()
    ctx.close()
    # the reference engine, whole converged fits, single thread
    eng_cls = checker.best_engine()
    kind = "reference" if eng_cls is checker.ReferenceEngine else "port"
    eng = eng_cls(d)
    eng.fit(MITTAL, 1e-6)
    reps, t_ref = 0, 0.0
    while t_ref < 2.0 and reps < 200:
        eng.set_beta(cold)
        t0 = time.perf_counter()
        ref_fit = eng.fit(MITTAL, 1e-6)
        t_ref += time.perf_counter() - t0
        reps += 1
    eng.close()
    port = checker.RestatementEngine(d)
    want = port.fit(MITTAL, 1e-6)
    port.close()
    active = active_columns(d)
    peak, peak_kind = read_peaks()
    total_bytes = sweep_bytes(d) * sweeps + objective_bytes(d) * (sweeps + attempts)
    scale = max(float(np.max(np.abs(want["beta"]))), 1e-8)
    line = {
        "metric": METRIC, "value": sweeps * active / dev_t, "unit": METRIC, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * dev_t / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded PCG64)",
        "config": {"workload": "logistic_l1", "model": "logistic", "rows": d.K, "columns": d.J, "nnz": d.nnz,
                   "prior": "laplace(0.1), none on the intercept", "convergence": "mittal (relative LL), tol 1e-6",
                   "precision": "fp64", "start": "cold (beta = 0)"},
        "step": "one converged findMode from a cold start",
        "time_to_converge_s": dev_t / args.steps,
        "sweeps_per_fit": sweeps / args.steps,
        "e2e": {"value": sweeps * active / e2e_t, "unit": METRIC, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d.J * 8)},
        "roofline": {"bound": "hbm", "achieved": total_bytes / ker_t / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": total_bytes / ker_t / 1e9 / peak, "peak_source": peak_kind,
                     "algorithmic_bytes_per_launch": total_bytes / attempts,
                     "kernel": ("resident_sweep_kernel<LOGISTIC> (one CTA, row state in shared memory)"
                                if args.strategy in ("auto", "resident") else
                                f"{args.strategy} sweep of the independent-row engine"), "traffic": None,
                     "note": "1.1e5 entries per sweep: latency-bound, L2-resident"},
        "cpu_baseline": {"value": ref_fit["iterations"] * active * reps / t_ref, "unit": METRIC, "cores": 1,
                         "kind": kind, "time_to_converge_s": t_ref / reps,
                         "sample": f"{reps} whole converged fits, single thread"},
        "parity": {"oracle": "FP64 restatement of the reference",
                   "max_rel_dbeta": float(np.max(np.abs(r.beta - want["beta"]))) / scale,
                   "rel_dll": abs(r.log_likelihood - want["loglik"]) / max(1.0, abs(want["loglik"])),
                   "iterations": {"gpu": int(r.iterations), "oracle": int(want["iterations"])},
                   "return_flag": {"gpu": int(r.return_flag), "oracle": int(want["flag"])}},
        "gpu_launches": int(launches), "clocks": clk,
    }
    if collect:
        return line
    print(json.dumps(line), flush=True)


def run_logistic_l1_reference(args, world, rank):
    """The reference engine on the CPU-runnable configuration: one whole
    converged fit per step (a few milliseconds), single thread."""
    if rank != 0:
        return
    from ccd_b200.data import MITTAL
    from oracle import checker
    d = synthetic.logistic_l1(seed=1)
    eng_cls = checker.best_engine()
    kind = "reference" if eng_cls is checker.ReferenceEngine else "port"
    eng = eng_cls(d)
    times, sweeps = [], 0
    for i in range(args.warmup + args.steps):
        eng.set_beta(cold_beta(d))
        t0 = time.perf_counter()
        r = eng.fit(MITTAL, 1e-6)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            times.append(dt)
            sweeps += r["iterations"]
    eng.close()
    total = float(np.sum(times))
    v = sweeps * active_columns(d) / total
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": METRIC, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded PCG64)",
        "config": {"workload": "logistic_l1", "model": "logistic", "rows": d.K, "columns": d.J, "nnz": d.nnz,
                   "prior": "laplace(0.1), none on the intercept", "convergence": "mittal (relative LL), tol 1e-6",
                   "precision": "fp64", "start": "cold (beta = 0)"},
        "step": "one converged findMode from a cold start",
        "time_to_converge_s": total / args.steps,
        "cpu_baseline": {"value": v, "unit": METRIC, "cores": 1, "kind": kind,
                         "sample": "one whole converged fit per step, single thread"},
        "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_extras(args, local) -> dict:
    """The other configurations, measured after the headline in the same run
    and nested in its line: the CPU-runnable L1 logistic fit, the Breslow Cox
    fit, the cross-validation grid and the served stream.  Each runs its own
    workload with a few warm-up and timed steps (bounded so the whole bench
    stays within minutes); a failure is recorded, not raised."""
    import copy
    global WORKLOAD
    out = {}
    plans = [
        ("logistic_l1", run_logistic_l1, dict(steps=max(3, min(args.steps, 20)), warmup=max(3, args.warmup))),
        ("cox_breslow", run_ours, dict(steps=1, warmup=1, no_cpu_baseline=args.no_cpu_baseline)),
        ("cv_grid", run_cv, dict(steps=1, warmup=1, plain_sample=2, fp64_check=2)),
        ("serve", run_serve, dict(steps=1, warmup=1, serve_requests=200)),
    ]
    for name, fn, over in plans:
        a = copy.copy(args)
        for k, v in over.items():
            setattr(a, k, v)
        a.workload = name
        WORKLOAD = name
        t0 = time.perf_counter()
        try:
            out[name] = fn(a, 1, 0, local, collect=True)
        except Exception as ex:  # recorded in the line
            out[name] = {"error": f"{type(ex).__name__}: {str(ex)[:300]}"}
        out[name]["bench_seconds"] = time.perf_counter() - t0
    WORKLOAD = "poisson_offset"
    return out


def cv_workload(small: bool, columns: int = 20_000):
    if small:
        d = synthetic.logistic_cv(seed=4, K=50_000, P=max(1, columns // 10))
    else:
        d = synthetic.logistic_cv(seed=4, P=columns)
    fold = synthetic.cv_folds(d.K, n_folds=10, seed=7)
    hold, var = synthetic.cv_grid(n_folds=10, n_vars=20, lower=1e-4, upper=1.0)
    return d, fold, hold, var


def cv_bytes(d, res) -> float:
    """Algorithmic bytes of a grid (the batched form of the per-coordinate count): column indices once for
    all instances (the most any instance gathered), per instance one 8-byte state word
    per gathered entry, 4-byte weight per entry, read+write per updated entry, and the
    convergence checks (y and xBeta per row per sweep)."""
    idx = max(r["gradient_entries"] for r in res) * 4.0
    per = sum(r["gradient_entries"] * (8.0 + 4.0) + r["update_entries"] * (4.0 + 16.0)
              + (r["iterations"] + 1) * d.K * 16.0 for r in res)
    return idx + per


def run_cv(args, world, rank, local, collect=False):
    import torch
    import torch.distributed as tdist
    if world > 1:  # instances shard over the ranks; no data-path collective
        import datetime
        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from ccd_b200 import native
    d, fold, hold, var = cv_workload(args.small, args.cv_columns)
    n_grid = len(var)
    if world > 1:
        mine = cv_shard(n_grid, world, rank)
        hold, var = hold[mine], var[mine]
    mixed = args.precision == "mixed"
    prec = native.PRECISION_MIXED if mixed else native.PRECISION_FP64
    ctx = native.Context(local)
    m = native.Matrix(ctx, d)
    f = native.Fit(ctx, m, d, precision=prec)
    margs = native.ModeFindingArguments(convergence_type=GRADIENT, tolerance=1e-6,
                                        max_iterations=args.max_sweeps)
    tuned = None
    group, cluster = args.group, args.cluster
    if mixed and not args.group:
        # the launch shape from one measured sweep per candidate (ccd_b200.tune), outside the timing
        from ccd_b200 import tune
        ch = tune.tune_batch(f, var, hold, fold, margs)
        group, cluster = ch.group, ch.cluster
        tuned = {"group": group, "cluster": cluster, "cached": ch.cached,
                 "one_sweep_seconds": {f"G{g}C{c}": v for (g, c), v in sorted(ch.seconds.items())}}
    grid = lambda fit: fit.batch_find_mode(var, hold, fold, margs, group=group, cluster=cluster)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=f"cuda:{local}")
    for _ in range(args.warmup):
        grid(f)
    clocks = Clocks(local)
    if world > 1:
        tdist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    t, fits, res_all, beta_all = 0.0, 0, None, None
    for _ in range(args.steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        beta, res, secs = grid(f)
        t += secs
        fits += len(var)
        res_all, beta_all = res, beta
    if world > 1:
        tdist.barrier()
    clk = clocks.stop()
    # whole job: every rank's fits over the slowest rank's device time
    t = allreduce([t], tdist.ReduceOp.MAX if world > 1 else None, world)[0]
    fits = int(allreduce([float(fits)], tdist.ReduceOp.SUM if world > 1 else None, world)[0])
    if world > 1 and rank != 0:
        tdist.barrier()
        tdist.destroy_process_group()
        return
    # end to end through the C ABI from host buffers: matrix upload, fit, coefficients back
    e2e_t = 0.0
    h2d = d.rows.nbytes + d.vals.nbytes + d.col_start.nbytes + d.val_start.nbytes + d.fmt.nbytes \
        + d.y.nbytes + fold.astype(np.int32).nbytes + var.nbytes + hold.astype(np.int32).nbytes
    d2h = len(var) * d.J * 8
    for _ in range(args.steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        me = native.Matrix(ctx, d)
        fe = native.Fit(ctx, me, d, precision=prec)
        grid(fe)
        e2e_t += time.perf_counter() - t0
        fe.close()
        me.close()
    # the plain solver on a sample of the same instances, one at a time
    plain_t, plain_n = 0.0, 0
    for i in np.linspace(0, len(var) - 1, args.plain_sample).astype(int):
        di = d.with_prior(1, float(var[i]))
        fi = native.Fit(ctx, m, di)
        fi.set_weights((fold != hold[i]).astype(float))
        r = fi.find_mode(native.ModeFindingArguments(convergence_type=GRADIENT, tolerance=1e-6,
                                                     max_iterations=args.max_sweeps))
        plain_t += r.device_seconds
        plain_n += 1
        fi.close()
    # error of the mixed engine against the FP64 engine on a sample of instances
    err = None
    if mixed and args.fp64_check > 0:
        idx = np.linspace(0, len(var) - 1, args.fp64_check).astype(int)
        f64 = native.Fit(ctx, m, d)
        b64, r64, _ = f64.batch_find_mode(var[idx], hold[idx], fold, margs)
        f64.close()
        ce = [float(np.max(np.abs(beta_all[i] - b64[q])) / max(np.max(np.abs(b64[q])), 1e-8))
              for q, i in enumerate(idx)]
        le = [abs(res_all[i]["loglik"] - r64[q]["loglik"]) / abs(r64[q]["loglik"]) for q, i in enumerate(idx)]
        err = {"instances": [int(i) for i in idx], "max_rel_coef": max(ce), "max_rel_loglik": max(le),
               "same_sweeps": int(sum(res_all[i]["iterations"] == r64[q]["iterations"] for q, i in enumerate(idx))),
               "fp64_engine": "FP64 batched engine (parity-tested against the reference CPU engine)"}
    cpu = None
    if not args.no_cpu_baseline:
        cpu = cv_cpu_sample(d, fold, hold, var, res_all)
    peak, peak_kind = read_peaks()
    byts = cv_bytes(d, res_all)
    achieved = byts / (t / args.steps) / 1e9
    sweeps = [r["iterations"] for r in res_all]
    kernel = "batch_mixed_kernel<LOGISTIC>" if mixed else "batch_sweep_kernel<LOGISTIC>"
    line = {
        "metric": "converged fits/s", "value": fits / t, "unit": "fits/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps,
        "higher_is_better": True, "scaling": "strong" if world > 1 else "weak", "vs_baseline": None,
        "dtype": "f32/f64 (f32 exp, ratios, per-entry terms; f64 state, reductions, step)" if mixed else "f64",
        "data": "synthetic (seeded PCG64, workload shapes of the benchmark config)",
        "config": cv_config(args, d, len(var), world),
        "launch_shape": tuned or {"group": group, "cluster": cluster or "engine's choice"},
        "e2e": {"value": world * len(var) * args.steps / e2e_t, "unit": "fits/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "plain_fits_per_s": plain_n / plain_t if plain_n else None,
        "batched_over_plain": (fits / t) / (plain_n / plain_t) if plain_n else None,
        "plain_sample": f"{plain_n} instances fitted one at a time by ccdb_find_mode (FP64)",
        "sweeps_per_fit": {"min": int(min(sweeps)), "median": float(np.median(sweeps)), "max": int(max(sweeps))},
        "error_vs_fp64": err,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind,
                     "algorithmic_bytes_per_launch": byts, "kernel": kernel,
                     "traffic": None},
        "cpu_baseline": cpu,
        "gpu_launches": args.steps,
        "clocks": clk,
    }
    f.close()
    m.close()
    ctx.close()
    if collect:
        return line
    print(json.dumps(line), flush=True)
    if world > 1:
        tdist.barrier()
        tdist.destroy_process_group()


def cv_config(args, d, instances: int, world: int) -> dict:
    """The cv_grid workload's config, the same on both arms."""
    return {"workload": "cv_grid" + ("_small" if args.small else "")
            + ("" if args.cv_columns == 20_000 else f"_{args.cv_columns}cols"), "model": "logistic",
            "rows": d.K, "columns": d.J, "nnz": d.nnz, "instances": instances,
            "folds": 10, "variances": "20 log-uniform in [1e-4, 1] (Laplace)",
            "convergence": "gradient, tol 1e-6", "start": "cold (beta = 0) per instance",
            "precision": args.precision, "group": args.group or "engine's choice",
            "parallelism": f"instances round-robin over {world} GPUs" if world > 1 else "1 GPU",
            "step": "one grid of 200 fits to convergence",
            "l2": "flushed between timed steps (512 MiB device write)"}


CV_REF_FOLDS = 4  # folds of the split the reference arm fits per step


def run_cv_reference(args, world, rank):
    """The reference's own cross-validation on the host cores: its
    GridSearchCrossValidationDriver (CcdInterface::runCrossValidation's grid
    path) with one host thread per fold task, on a bounded sample of the grid: at the
    smallest variance, the first 4 folds of the 10-fold split
    (foldToCompute = 4), then the refit on all rows.  Those are the grid's
    cheapest fits (the fewest sweeps), so the sample overstates the
    reference's throughput on the whole grid."""
    if rank != 0:
        return
    from oracle import checker
    d, fold, hold, var = cv_workload(args.small, args.cv_columns)
    lo = float(np.min(var))
    # one thread per fold task: the driver clones the engine for every thread
    # it is given, and more threads than tasks only add clones
    threads = min(os.cpu_count() or 1, CV_REF_FOLDS)
    eng_cls = checker.best_engine()
    kind = "reference" if eng_cls is checker.ReferenceEngine else "port"
    eng = eng_cls(d.with_prior(1, lo))
    times = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        if kind == "reference":
            eng.cross_validate(auto_search=False, fold=10, grid_steps=1, lower=lo, upper=lo, seed=7,
                               threads=threads, fold_to_compute=CV_REF_FOLDS)
        else:  # the oracle port has no driver: the same fits one after another
            for h in range(CV_REF_FOLDS):
                eng.set_weights((fold != h).astype(float))
                eng.set_beta(cold_beta(d))
                eng.fit(GRADIENT, 1e-6)
            eng.set_weights(None)
            eng.set_beta(cold_beta(d))
            eng.fit(GRADIENT, 1e-6)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            times.append(dt)
    eng.close()
    total = float(np.sum(times))
    v = (CV_REF_FOLDS + 1) * args.steps / total
    sample = (f"per step: {CV_REF_FOLDS} of the 10 fold fits at the grid's smallest variance ({lo:g}) and "
              f"the refit on all "
              f"rows, {'the reference GridSearchCrossValidationDriver on ' + str(threads) + ' threads' if kind == 'reference' else 'one thread'}; "
              f"the grid's cheapest fits, so this overstates the reference on the whole grid")
    line = {
        "impl": "reference", "metric": "converged fits/s", "value": v, "unit": "fits/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded PCG64, workload shapes of the benchmark config)",
        "config": cv_config(args, d, len(var), 1),
        "cpu_baseline": {"value": v, "unit": "fits/s", "cores": threads if kind == "reference" else 1,
                         "kind": kind, "sample": sample},
        "e2e": {"value": v, "unit": "fits/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def cv_cpu_sample(d, fold, hold, var, res):
    """The reference CPU engine on a bounded sample of the grid: the first sweep of
    the median-variance instance, single thread; fits/s = 1 / (that sweep time x the
    mean sweeps per fit the grid needed)."""
    from oracle import checker
    eng_cls = checker.best_engine()
    kind = "reference" if eng_cls is checker.ReferenceEngine else "port"
    i = len(var) // 2
    di = d.with_prior(1, float(var[i]))
    e = eng_cls(di)
    e.set_weights((fold != hold[i]).astype(float))
    t0 = time.perf_counter()
    e.fit(GRADIENT, 1e-6, 1)
    t_sweep = time.perf_counter() - t0
    e.close()
    mean_sweeps = float(np.mean([r["iterations"] for r in res]))
    return {"value": 1.0 / (t_sweep * mean_sweeps), "unit": "fits/s", "cores": 1, "kind": kind,
            "sample": f"first sweep of instance {i} (variance {var[i]:.3g}), {t_sweep:.2f} s, "
                      f"x {mean_sweeps:.1f} mean sweeps per fit of this grid, single thread"}


SERVE_RANGES = dict(rate=50.0, K_range=(1e3, 1e5), J_range=(1e2, 1e4), density_range=(0.001, 0.02))


def run_serve(args, world, rank, local, collect=False):
    """The served stream: Poisson(50/s) arrivals of independent logistic /
    conditional logistic / Cox fits, replayed in real time into the server."""
    import torch
    from ccd_b200 import native, serve
    if world > 1 and rank != 0:
        return  # one server per GPU box; replicas add nothing to a latency figure
    stream = synthetic.serving_stream(args.serve_requests, seed=11, **SERVE_RANGES)
    # warm-up requests of every kind the trace holds (logistic fits on the resident and
    # the cluster sweep, conditional logistic and Cox fits), so that each kernel has run once
    warm = synthetic.serving_stream(max(16, args.serve_slots + args.serve_fast_slots), seed=12, rate=1e3,
                                    K_range=(1e3, 3e4), J_range=(50, 200))
    srv = serve.Server(device=local, hbm_budget=150e9, slots=args.serve_slots, fast_slots=args.serve_fast_slots,
                       fast_ctas=args.serve_fast_ctas, slot_ctas=args.serve_slot_ctas)
    try:
        for _ in range(args.warmup):
            srv.done.clear()
            serve.replay(srv, warm)
        clocks = Clocks(local)
        torch.cuda.synchronize()
        clocks.start()
        summaries = []
        for _ in range(args.steps):
            srv.done.clear()
            done = serve.replay(srv, stream)
            summaries.append(serve.latency_summary(done))
        # service time (start to end) per model type: where the GPU time goes
        svc = collections.defaultdict(list)
        for c in done:
            svc[int(stream[c.rid][1].model_type)].append(c.end - c.start)
        service = {str(k): {"n": len(v), "median_s": float(np.median(v)), "max_s": float(np.max(v))}
                   for k, v in sorted(svc.items())}
        errors = collections.Counter(
            f"model {int(stream[c.rid][1].model_type)}: {c.error[:160]}" for c in done if c.error)
        # the requests the reference arm's sample serves, within this whole replay
        head = np.array([c.latency for c in done if c.rid < SERVE_REF_REQUESTS])
        clk = clocks.stop()
        peak = srv.peak_running
    finally:
        srv.close()
    if args.serve_detail:
        # per-request timeline of the last replay, and each request fitted alone on a
        # context limited like the slot that served it (outside the timed region)
        recs = serve.request_records(stream, done)
        ctxs = {}
        try:
            for r in recs:
                lim = srv.slot_max_ctas(r["slot"], torch.cuda.get_device_properties(local).multi_processor_count)
                if lim not in ctxs:
                    ctxs[lim] = native.Context(local)
                    ctxs[lim].set_max_ctas(lim)
                t0 = time.perf_counter()
                native.fit_model(ctxs[lim], stream[r["rid"]][1], native.ModeFindingArguments())
                r["alone_s"] = time.perf_counter() - t0
        finally:
            for c in ctxs.values():
                c.close()
        with open(args.serve_detail, "w") as fh:
            for r in recs:
                fh.write(json.dumps(r) + "\n")
    s = summaries[-1]
    h2d = sum(d.rows.nbytes + d.vals.nbytes + d.col_start.nbytes + d.val_start.nbytes + d.y.nbytes
              + (d.time.nbytes if d.time is not None else 0) + (d.stratum.nbytes if d.stratum is not None else 0)
              for _, d in stream)
    d2h = sum(8 * d.J for _, d in stream)
    cpu = None if args.no_cpu_baseline else serve_cpu_sample(stream)
    line = {
        "metric": "p50 fit latency", "value": s["p50_s"], "unit": "s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * s["makespan_s"], "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded PCG64 problems and arrival trace)",
        "config": serve_config(args, stream),
        "p99_s": s["p99_s"], "mean_s": s["mean_s"], "fits_per_s": s["fits_per_s"],
        "failed": s["failed"], "errors": dict(errors.most_common(5)), "peak_concurrent_fits": peak,
        "service_by_model": service,
        "first_requests": {"n": int(head.size), "p50_s": float(np.percentile(head, 50)),
                           "p99_s": float(np.percentile(head, 99)),
                           "note": "the first requests of the trace (the reference arm's sample), "
                                   "served within the whole replay"},
        "e2e": {"value": s["p50_s"], "unit": "s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "roofline": None, "cpu_baseline": cpu, "gpu_launches": None, "clocks": clk,
    }
    if collect:
        return line
    print(json.dumps(line), flush=True)


def serve_config(args, stream) -> dict:
    """The serve workload's config, the same on both arms."""
    kinds = collections.Counter(int(d.model_type) for _, d in stream)
    return {"workload": "serve", "requests": len(stream), "arrivals": "Poisson, 50/s",
            "mix": {str(k): v for k, v in sorted(kinds.items())},
            "K": "log-uniform 1e3..1e5", "J": "log-uniform 1e2..1e4",
            "density": "uniform 0.001..0.02", "prior": "Laplace, variance 0.1",
            "slots": args.serve_slots, "fast_slots": args.serve_fast_slots, "fast_slot_ctas": args.serve_fast_ctas,
            "slot_ctas": args.serve_slot_ctas or "even share",
            "fast_lane": "requests of at most 200,000 matrix entries, oldest first",
            "hbm_budget_bytes": 150e9,
            "step": "replay of the whole stream; latency = completion - arrival",
            "strategy": "logistic: the resident sweep (one CTA) when the rows fit it, else the "
                        "cluster sweep on the slot's share of the SMs; grouped models: the group sweep"}


def _serve_cpu_latencies(stream, n: int):
    """Latencies of the reference CPU engine serving the first n requests of
    the trace: FIFO over a pool of all host cores, each fit single-threaded,
    replayed at the trace's arrival times."""
    import concurrent.futures as cf
    from oracle import checker
    eng_cls = checker.best_engine()
    kind = "reference" if eng_cls is checker.ReferenceEngine else "port"
    sub = stream[:n]
    cores = os.cpu_count() or 1

    def one(d):
        e = eng_cls(d)
        try:
            e.fit(GRADIENT, 1e-6, 1000)
        finally:
            e.close()
        return time.perf_counter()

    t0 = time.perf_counter()
    futs = []
    with cf.ThreadPoolExecutor(max_workers=cores) as ex:
        for t_arr, d in sub:
            delay = t0 + t_arr - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            futs.append((t0 + t_arr, ex.submit(one, d)))
        lat = np.array([f.result() - a for a, f in futs])
    return lat, cores, kind


def serve_cpu_sample(stream, n: int = 40):
    """The reference CPU engine serving the first n requests of the same trace
    (the GPU line's cpu_baseline)."""
    lat, cores, kind = _serve_cpu_latencies(stream, n)
    return {"value": float(np.percentile(lat, 50)), "unit": "s", "cores": cores, "kind": kind,
            "p99_s": float(np.percentile(lat, 99)),
            "sample": f"first {len(lat)} requests of the same trace, FIFO over {cores} host threads"}


SERVE_REF_REQUESTS = 40  # requests of the trace the reference arm serves per step


def run_serve_reference(args, world, rank):
    """The reference CPU engine serving the same seeded trace: per step the
    first 40 requests, replayed at their arrival times, FIFO over a pool of
    all host cores (each fit single-threaded, as the reference's inner loop
    is serial); the p50 latency over the timed steps' requests."""
    if rank != 0:
        return
    stream = synthetic.serving_stream(args.serve_requests, seed=11, **SERVE_RANGES)
    lats, spans, cores, kind = [], [], 1, "port"
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        lat, cores, kind = _serve_cpu_latencies(stream, SERVE_REF_REQUESTS)
        if i >= args.warmup:
            lats.extend(lat.tolist())
            spans.append(time.perf_counter() - t0)
    p50 = float(np.percentile(lats, 50))
    line = {
        "impl": "reference", "metric": "p50 fit latency", "value": p50, "unit": "s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(spans)),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded PCG64 problems and arrival trace)", "config": serve_config(args, stream),
        "p99_s": float(np.percentile(lats, 99)),
        "cpu_baseline": {"value": p50, "unit": "s", "cores": cores, "kind": kind,
                         "sample": f"per step the first {SERVE_REF_REQUESTS} of the trace's {len(stream)} "
                                   f"requests, FIFO over {cores} host threads"},
        "e2e": {"value": p50, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ variants
VARIANTS = ("kkt_l1", "mm_clr", "fisher_l1")
STRATEGIES = {"auto": 0, "levels": 1, "speculative": 2, "grid_levels": 3, "resident": 4}


def variant_problem(name: str):
    """kkt_l1: L1 logistic regression on the cross-validation grid's shared
    matrix (500,000 rows x 20,000 indicator covariates at density 0.005, ~5e7
    nonzeros, intercept) with Laplace variance 0.01 -- a sparse fit, the case
    the swindle is for; mm_clr: conditional logistic regression, 50,000 matched
    sets of 2-11 rows (~325,000 rows), 5,000 indicator covariates at density
    0.01, Laplace variance 0.1; fisher_l1: the 10,000 x 1,000 L1 logistic
    problem (density 0.01, intercept, Laplace variance 0.1), information over
    all 1,001 columns at its mode."""
    if name == "mm_clr":
        return synthetic.conditional_logistic(seed=5, n_sets=50_000, P=5_000)
    if name == "kkt_l1":
        d = synthetic.logistic_cv(seed=4)
        d.prior_var[:] = 0.01
        return d
    return synthetic.logistic_l1(seed=1)


def variant_fit_kw(name: str) -> dict:
    """Oracle / reference fit() keywords and the matching C ABI mode arguments."""
    if name == "kkt_l1":
        return dict(kkt_swindle=True)
    if name == "mm_clr":
        return dict(algorithm=1)
    return {}


def variant_config(name: str, d) -> dict:
    from ccd_b200.data import MITTAL  # noqa: F401 (documented below)
    base = {"workload": name, "rows": d.K, "columns": d.J, "nnz": d.nnz, "precision": "fp64",
            "prior": f"laplace({float(d.prior_var[-1]):g}), none on the intercept",
            "convergence": "relative log-likelihood change (mittal), tol 1e-6",
            "l2": "flushed between timed steps (512 MiB device write)"}
    if name == "kkt_l1":
        return {**base, "model": "logistic", "step": "one converged KKT-swindle fit from a cold start"}
    if name == "mm_clr":
        return {**base, "model": "conditional logistic", "strata": int(d.stratum.max()) + 1,
                "step": "one converged MM fit from a cold start"}
    return {**base, "model": "logistic", "step": "Fisher information over every coefficient column "
                                                 "at the fitted mode (n = columns)"}


def variant_unit(name: str) -> str:
    return "Fisher entries/s" if name == "fisher_l1" else "fits/s"


def fisher_cols(d) -> np.ndarray:
    return np.arange(1 if d.offset_col0 else 0, d.J, dtype=np.int32)


def fisher_bytes(d, cols) -> float:
    """Algorithmic bytes of one Fisher call: per pass of 8 columns, the scatter
    reads each of its columns' entries (row id 4 B where stored, value 8 B where
    stored) and writes an 8-byte table slot; the gather reads, per entry of every
    column at or after the pass, the row id / value, a 64-byte table row and
    the 32-byte row state."""
    n = len(cols)
    ent = np.array([d.K if d.fmt[j] in (DENSE, INTERCEPT) else d.col_start[j + 1] - d.col_start[j]
                    for j in cols], dtype=np.float64)
    per = np.array([(4 if d.fmt[j] in (SPARSE, INDICATOR) else 0) + (8 if d.fmt[j] in (SPARSE, DENSE) else 0)
                    for j in cols], dtype=np.float64)
    suffix = np.cumsum((ent * (per + 64 + 32))[::-1])[::-1]
    total = 0.0
    for p0 in range(0, n, 8):
        total += float(np.sum(ent[p0:p0 + 8] * (per[p0:p0 + 8] + 8))) + float(suffix[p0])
    return total


def mm_cycle_bytes(d) -> float:
    """Algorithmic bytes of one MM cycle's bound kernel: per entry the row id
    (4 B) and value (8 B where stored), {xBeta, e} (16 B), the group (4 B), the
    group's events and denominator (16 B)."""
    cnt = np.diff(d.col_start).astype(np.float64)
    val = np.where((d.fmt == SPARSE) | (d.fmt == DENSE), 8.0, 0.0)
    return float(np.sum(cnt * (4 + val + 16 + 4 + 16)))


def variant_reference_time(eng, name: str, d, cols) -> float:
    """Seconds of one step of the reference CPU engine (single thread)."""
    from ccd_b200.data import MITTAL
    if name == "fisher_l1":
        t0 = time.perf_counter()
        eng.fisher_information(cols)
        return time.perf_counter() - t0
    eng.set_beta(cold_beta(d))
    t0 = time.perf_counter()
    eng.fit(MITTAL, 1e-6, **variant_fit_kw(name))
    return time.perf_counter() - t0


def variant_reference_engine(name: str, d):
    from ccd_b200.data import MITTAL
    from oracle import checker
    eng_cls = checker.best_engine()
    kind = "reference" if eng_cls is checker.ReferenceEngine else "port"
    eng = eng_cls(d)
    if name == "fisher_l1":
        eng.fit(MITTAL, 1e-6)  # the state the information is taken at
    return eng, kind


def variant_units_per_step(name: str, d) -> float:
    if name == "fisher_l1":
        n = len(fisher_cols(d))
        return n * (n + 1) / 2.0
    return 1.0


def run_variant_reference(args, world, rank):
    if rank != 0:
        return
    d = variant_problem(args.workload)
    cols = fisher_cols(d)
    eng, kind = variant_reference_engine(args.workload, d)
    times = []
    for i in range(args.warmup + args.steps):
        dt = variant_reference_time(eng, args.workload, d, cols)
        if i >= args.warmup:
            times.append(dt)
    eng.close()
    total = float(np.sum(times))
    unit = variant_unit(args.workload)
    v = args.steps * variant_units_per_step(args.workload, d) / total
    line = {
        "impl": "reference", "metric": unit, "value": v, "unit": unit, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded PCG64)", "config": variant_config(args.workload, d),
        "cpu_baseline": {"value": v, "unit": unit, "cores": 1, "kind": kind,
                         "sample": "the whole step per step, single thread"},
        "e2e": {"value": v, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_variant(args, world, rank, local):
    """The KKT swindle, the MM algorithm or the Fisher information; each rank
    runs its own replica (these fits do not shard)."""
    import torch
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    import torch.distributed as tdist
    from ccd_b200 import native
    from ccd_b200.data import MITTAL
    name = args.workload
    d = variant_problem(name)
    cols = fisher_cols(d)
    ctx = native.Context(local)
    m = native.Matrix(ctx, d)
    f = native.Fit(ctx, m, d)
    kw = variant_fit_kw(name)
    margs = native.ModeFindingArguments(convergence_type=MITTAL, tolerance=1e-6,
                                        max_iterations=args.max_sweeps,
                                        algorithm=kw.get("algorithm", 0),
                                        kkt_swindle=kw.get("kkt_swindle", False),
                                        strategy=STRATEGIES[args.strategy])
    cold = cold_beta(d)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=f"cuda:{local}")
    units = variant_units_per_step(name, d)
    if name == "fisher_l1":
        f.set_beta(cold)
        fitted = f.find_mode(margs)

    def one_step():
        """Device seconds, launches and cycles of one step."""
        if name == "fisher_l1":
            f.compute_fisher_information(cols)
            return f.last_call_seconds(), 2 * ((len(cols) + 7) // 8), 1
        f.set_beta(cold)
        r = f.find_mode(margs)
        return r.device_seconds, r.kernel_launches, r.iterations

    for _ in range(args.warmup):
        one_step()
    clocks = Clocks(local)
    if world > 1:
        tdist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    dev_t, launches, cycles = 0.0, 0, 0
    for _ in range(args.steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        t, nl, it = one_step()
        dev_t += t
        launches += nl
        cycles += it
    torch.cuda.synchronize()
    clk = clocks.stop()

    # end to end from host buffers: the one-call fit (upload, fit, beta back) or
    # the Fisher call with its index upload and n x n copy back, host-timed
    if name == "fisher_l1":
        h2d, d2h = len(cols) * 4, len(cols) ** 2 * 8
        e2e_t = 0.0
        for _ in range(args.steps):
            flush.fill_(1)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            f.compute_fisher_information(cols)
            e2e_t += time.perf_counter() - t0
    else:
        def pinned(a):
            return torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
        from ccd_b200.data import CyclopsData
        dp = CyclopsData(d.model_type, pinned(d.y), pinned(d.col_start), pinned(d.rows),
                         pinned(d.val_start), pinned(d.vals), pinned(d.fmt), d.prior_type, d.prior_var,
                         time=d.time, stratum=d.stratum, offset_col0=d.offset_col0)
        h2d = sum(a.nbytes for a in (dp.y, dp.col_start, dp.rows, dp.val_start, dp.vals, dp.fmt))
        d2h = d.J * 8
        e2e_t = 0.0
        for _ in range(args.steps):
            flush.fill_(1)
            torch.cuda.synchronize()
            e2e_t += native.fit_model(ctx, dp, margs).device_seconds
    mx = allreduce([dev_t, e2e_t], tdist.ReduceOp.MAX if world > 1 else None, world)
    sm = allreduce([float(launches)], tdist.ReduceOp.SUM if world > 1 else None, world)
    if rank == 0:
        unit = variant_unit(name)
        peak, peak_kind = read_peaks()
        roofline = None
        if name == "fisher_l1":
            b = fisher_bytes(d, cols)
            ach = b * args.steps / dev_t / 1e9
            roofline = {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                        "peak_source": peak_kind, "algorithmic_bytes_per_launch": b / (2 * ((len(cols) + 7) // 8)),
                        "kernel": "fisher_scatter + fisher_gather passes (one call)", "traffic": None}
        elif name == "mm_clr":
            b = mm_cycle_bytes(d) * cycles
            ach = b / dev_t / 1e9
            roofline = {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                        "peak_source": peak_kind, "algorithmic_bytes_per_launch": mm_cycle_bytes(d),
                        "kernel": "mm_gh_kernel (bound of one cycle; timed over the whole fit)",
                        "traffic": None}
        line = {
            "metric": unit, "value": world * args.steps * units / mx[0], "unit": unit, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * mx[0] / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded PCG64)",
            "config": {**variant_config(name, d), "parallelism": f"replicas x{world}",
                       "sweep_strategy": args.strategy},
            "cycles_per_step": cycles / args.steps,
            "e2e": {"value": world * args.steps * units / mx[1], "unit": unit,
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
            "roofline": roofline,
            "gpu_launches": int(sm[0]),
            "clocks": clk,
        }
        if name == "fisher_l1":
            line["fitted"] = {"iterations": fitted.iterations, "return_flag": fitted.return_flag}
        if world == 1 and not args.no_cpu_baseline:
            eng, kind = variant_reference_engine(name, d)
            t = variant_reference_time(eng, name, d, cols)
            eng.close()
            line["cpu_baseline"] = {"value": units / t, "unit": unit, "cores": 1, "kind": kind,
                                    "sample": f"one whole step ({t:.2f} s), single thread"}
        print(json.dumps(line), flush=True)
    f.close()
    m.close()
    ctx.close()
    if world > 1:
        tdist.destroy_process_group()


def main():
    global WORKLOAD
    args = parse()
    WORKLOAD = args.workload
    world, rank, local = dist_setup()
    if args.impl == "reference" and args.workload in VARIANTS:
        run_variant_reference(args, world, rank)
    elif args.impl == "reference" and args.workload == "cv_grid":
        run_cv_reference(args, world, rank)
    elif args.impl == "reference" and args.workload == "serve":
        run_serve_reference(args, world, rank)
    elif args.impl == "reference" and args.workload == "logistic_l1":
        run_logistic_l1_reference(args, world, rank)
    elif args.impl == "reference":
        run_reference(args, world, rank)
    elif args.workload in VARIANTS:
        run_variant(args, world, rank, local)
    elif args.workload == "cv_grid":
        run_cv(args, world, rank, local)
    elif args.workload == "serve":
        run_serve(args, world, rank, local)
    elif args.workload == "logistic_l1":
        run_logistic_l1(args, world, rank, local)
    else:
        run_ours(args, world, rank, local)


if __name__ == "__main__":
    main()
