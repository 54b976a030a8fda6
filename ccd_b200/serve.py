"""Serving: a request loop over independent fits with continuous batching.

Requests (a problem and its mode-finding arguments) arrive over time.  A
fixed set of slots -- host threads, each with its own engine context and so
its own CUDA stream -- takes requests in arrival order as soon as a slot is
free and the request's device-memory estimate fits the HBM budget next to the
fits already running; a request that arrives while others are on the GPU is
admitted the moment a slot and memory free up, and its kernels overlap theirs
on the device.  A fit runs exactly as it would alone (same engine, same
kernels, same arithmetic: its result does not depend on its neighbours); the
server only decides when it starts.

Each slot's context limits its sweep kernels to its share of the SMs (a
fast slot one CTA, a general slot an even share of the rest), so the slots'
kernels can all be resident at once and run side by side.  Every model runs
a whole findMode attempt in one launch: logistic and Poisson fits whose row
state fits one CTA's shared memory the resident sweep (one CTA), larger ones
the cluster sweep over dependency levels (a thread block cluster of at most
that many CTAs), grouped models (conditional logistic, Cox) the persistent
group sweep (a cluster, or a cooperative grid, of at most that many CTAs).

The reference has no serving layer; this loop drives the same C ABI entry
point a single fit uses (ccdb_fit_model: upload, findMode, coefficients back).
"""
from __future__ import annotations

import collections
import threading
import time
from dataclasses import dataclass
from typing import Callable, List, Optional

import numpy as np

from .data import CyclopsData


@dataclass
class Request:
    rid: int
    data: CyclopsData
    args: object = None          # native.ModeFindingArguments (None: the defaults)
    bytes: int = 0               # device-memory estimate used for admission
    arrival: float = 0.0         # time.perf_counter() at submission


@dataclass
class Completed:
    rid: int
    beta: np.ndarray
    flag: int
    iterations: int
    loglik: float
    arrival: float
    start: float
    end: float
    slot: int
    error: Optional[str] = None

    @property
    def latency(self) -> float:
        return self.end - self.arrival


def estimate_bytes(d: CyclopsData) -> int:
    """Upper estimate of a fit's device memory: the matrix (CSC and the CSR copy
    a warm start may build), the per-row state, per-column state and, for Cox,
    the risk-set tables; twice that for allocator slack and a fixed 64 MiB."""
    nnz, nv = int(d.nnz), int(d.vals.size)
    core = 12 * nnz + 8 * nv + 16 * (d.J + 1) + 96 * d.K + 96 * d.J
    if d.time is not None:
        core += 120 * d.K
    return 2 * core + (64 << 20)


def is_small(d: CyclopsData, max_entries: int) -> bool:
    """A request the fast lane may take: at most max_entries matrix entries
    (dense-like columns count K each)."""
    return int(d.nnz) <= max_entries


class Server:
    """`slots` concurrent fits under an HBM budget of `hbm_budget` bytes, plus
    `fast_slots` slots that take only small requests (at most `fast_entries`
    matrix entries) on at most `fast_ctas` CTAs each; a general slot's fits
    take at most `slot_ctas` CTAs (0: an even share of the SMs the fast slots
    leave).

    The general slots take requests in arrival order (no overtaking).  A fast
    slot takes the oldest pending small request, ahead of any large one: a
    small fit takes milliseconds, a large one seconds, and without the lane a
    burst of large requests holds every slot while the small ones queue.
    Within each class the order of arrival is kept.

    ``fit_fn(slot, request, slot_state) -> (beta, flag, iterations, loglik)``
    runs one fit (`slot_state` is the slot thread's own attribute holder); the
    default runs it on the GPU through the slot's own context.  Tests of the
    admission logic pass a stand-in that needs no GPU.
    """

    def __init__(self, device: int = 0, hbm_budget: float = 150e9, slots: int = 8,
                 fit_fn: Optional[Callable] = None, fast_slots: int = 0, fast_entries: int = 200_000,
                 fast_ctas: int = 1, slot_ctas: int = 0):
        self.device = device
        self.budget = int(hbm_budget)
        self.n_slots = slots
        self.n_fast = fast_slots
        self.fast_entries = int(fast_entries)
        self.fast_ctas = max(1, int(fast_ctas))
        self.slot_ctas = max(0, int(slot_ctas))  # 0: the SMs the fast slots leave, shared evenly
        self._fit_fn = fit_fn or self._gpu_fit
        self._cv = threading.Condition()
        self._pending: collections.deque = collections.deque()
        self._reserved = 0
        self._running = 0
        self._stop = False
        self.peak_reserved = 0
        self.peak_running = 0
        self.done: List[Completed] = []
        self._threads = [threading.Thread(target=self._worker, args=(i,), daemon=True)
                         for i in range(slots + fast_slots)]
        for t in self._threads:
            t.start()

    # -- submission and shutdown
    def submit(self, req: Request) -> None:
        if not req.bytes:
            req.bytes = estimate_bytes(req.data)
        if req.bytes > self.budget:
            raise ValueError(f"request {req.rid} needs ~{req.bytes} bytes, above the HBM budget {self.budget}")
        req.arrival = time.perf_counter()
        with self._cv:
            self._pending.append(req)
            self._cv.notify_all()

    def drain(self, n_expected: int, timeout: float = 3600.0) -> List[Completed]:
        """Wait until n_expected requests have completed."""
        t_end = time.perf_counter() + timeout
        with self._cv:
            while len(self.done) < n_expected:
                left = t_end - time.perf_counter()
                if left <= 0:
                    raise TimeoutError(f"{len(self.done)} of {n_expected} requests completed")
                self._cv.wait(min(left, 1.0))
            return list(self.done)

    def close(self) -> None:
        with self._cv:
            self._stop = True
            self._cv.notify_all()
        for t in self._threads:
            t.join()

    # -- the slots
    def _next(self, fast: bool):
        """Index of the request this slot may admit now, or None."""
        if not fast:
            if self._pending and self._reserved + self._pending[0].bytes <= self.budget:
                return 0  # the oldest request fits: admit it (arrival order)
            return None
        for i, r in enumerate(self._pending):  # the oldest small request that fits
            if is_small(r.data, self.fast_entries):
                return i if self._reserved + r.bytes <= self.budget else None
        return None

    def _worker(self, slot: int) -> None:
        local = threading.local()
        fast = slot >= self.n_slots
        if self._fit_fn == self._gpu_fit:  # the slot's context exists before its first request
            try:
                self._gpu_slot_init(slot, local)
            except Exception:  # retried by the first request, which then fails with the error
                ctx = local.__dict__.pop("ctx", None)
                if ctx is not None:
                    try:
                        ctx.close()
                    except Exception:
                        pass
        while True:
            with self._cv:
                while True:
                    i = self._next(fast)
                    if i is not None:
                        break
                    if self._stop and not self._pending:
                        ctx = getattr(local, "ctx", None)
                        if ctx is not None:
                            ctx.close()
                        return
                    self._cv.wait()
                req = self._pending[i]
                del self._pending[i]
                self._reserved += req.bytes
                self._running += 1
                self.peak_reserved = max(self.peak_reserved, self._reserved)
                self.peak_running = max(self.peak_running, self._running)
            start = time.perf_counter()
            beta, flag, iters, ll, err = None, -1, 0, float("nan"), None
            try:
                beta, flag, iters, ll = self._fit_fn(slot, req, local)
            except Exception as e:  # the request fails, the server keeps serving
                err = f"{type(e).__name__}: {e}"
            end = time.perf_counter()
            with self._cv:
                self._reserved -= req.bytes
                self._running -= 1
                self.done.append(Completed(req.rid, beta, flag, iters, ll, req.arrival, start, end, slot, err))
                self._cv.notify_all()

    def slot_max_ctas(self, slot: int, n_sm: int) -> int:
        """The CTA limit of a slot's context on a GPU of n_sm SMs.

        General slots share the SMs the fast slots leave (at most slot_ctas
        each when set); a fast slot's small fits run on fast_ctas CTAs (default
        one: the resident sweep, or a one-CTA cluster or group sweep), which
        find a free SM beside the general slots' clusters, where a multi-CTA
        cluster may have to wait for a whole GPC."""
        if slot >= self.n_slots:
            return self.fast_ctas
        general = max(1, (n_sm - self.n_fast * self.fast_ctas) // max(1, self.n_slots))
        return min(general, self.slot_ctas) if self.slot_ctas else general

    def _gpu_slot_init(self, slot: int, local) -> None:
        from . import native
        local.ctx = native.Context(self.device)
        local.ctx.set_max_ctas(self.slot_max_ctas(slot, local.ctx.sm_count))
        local.ctx.set_blocking_wait(True)  # slots wait without spinning the host cores

    def _gpu_fit(self, slot: int, req: Request, local):
        from . import native
        if not hasattr(local, "ctx"):
            self._gpu_slot_init(slot, local)
        args = req.args or native.ModeFindingArguments()
        r = native.fit_model(local.ctx, req.data, args)
        return r.beta, r.return_flag, r.iterations, r.log_likelihood


def replay(server: Server, stream, args=None, time_scale: float = 1.0) -> List[Completed]:
    """Submit [(arrival seconds, CyclopsData)] at their arrival times and wait for
    every result.  Returns the completions in request order."""
    t0 = time.perf_counter()
    for i, (t_arr, d) in enumerate(stream):
        delay = t0 + t_arr * time_scale - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        server.submit(Request(i, d, args))
    done = server.drain(len(stream))
    return sorted(done, key=lambda c: c.rid)


def request_records(stream, done: List[Completed]) -> List[dict]:
    """One record per completed request of a replay of `stream` ([(arrival
    seconds, CyclopsData)]): its model, size, slot, and the wait (arrival to
    start) and service (start to end) times, with the start and end as offsets
    from the first arrival -- the timeline in which fits held up by their
    neighbours show as service times far above their time alone."""
    if not done:
        return []
    first = min(c.arrival for c in done)
    out = []
    for c in sorted(done, key=lambda c: c.rid):
        d = stream[c.rid][1]
        out.append({"rid": int(c.rid), "model": int(d.model_type), "K": int(d.K), "J": int(d.J),
                    "entries": int(d.nnz), "slot": int(c.slot), "arrival_s": c.arrival - first,
                    "start_s": c.start - first, "end_s": c.end - first, "wait_s": c.start - c.arrival,
                    "service_s": c.end - c.start, "flag": int(c.flag), "error": c.error})
    return out


def latency_summary(done: List[Completed]) -> dict:
    lat = np.array([c.latency for c in done])
    first = min(c.arrival for c in done)
    last = max(c.end for c in done)
    return {"requests": len(done), "failed": sum(c.error is not None for c in done),
            "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "fits_per_s": len(done) / (last - first),
            "makespan_s": last - first}
