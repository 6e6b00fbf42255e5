"""Serving loop over resident tables: continuous batching with HBM-budget
admission and the learned sizer.

Requests (mixed-workload queries) arrive as a Poisson process. Worker
threads, each with its own batch object (own CUDA stream, own device
arena), repeatedly take every request that has arrived and fits the HBM
budget, run them as one batch through the batched, learned-sizing path and
hand back the results; while one worker's batch is on the GPU the next
worker is already admitting the requests that arrived meanwhile, so their
work overlaps on the device. The C calls release the GIL, so the workers
run concurrently.

The reference has no serving layer (one query per process invocation,
codegen/codegen_main.cpp:384-405); the one-query-at-a-time baseline here is
the plain engine path (PlainRunner) behind a FIFO queue.
"""
from __future__ import annotations

import math
import threading
import time
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import batch as B


@dataclass
class Request:
    id: int
    query: B.MixQuery
    arrival: float  # seconds after the start of the trace


def poisson_trace(queries: Sequence[B.MixQuery], rate: float, seed: int = 0) -> List[Request]:
    """Requests for `queries` with exponential inter-arrival times (mean
    1 / rate seconds)."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, len(queries)))
    return [Request(i, q, float(t[i])) for i, q in enumerate(queries)]


def query_hbm_bytes(q: B.MixQuery, dim_max_key: int) -> int:
    """Upper bound of the device memory one query of a batch can take:
    its hash table sized for min(card, rows) groups (the learned size is
    never larger), slot list, collected rows and join bitmap."""
    if q.grouped:
        slots = 1 << max(4, math.ceil(math.log2(2 * max(1, min(q.card, q.rows)))))
        return slots * (16 + 4 + 24) + 4096
    if q.tmpl == "join":
        return dim_max_key // 8 + 4096
    return 4096


@dataclass
class ServeReport:
    rate: float
    requests: int
    wall_s: float
    latencies_s: np.ndarray
    batches: int
    batch_sizes: List[int] = field(default_factory=list)
    overflowed: int = 0
    peak_reserved_bytes: int = 0
    overlap_s: float = 0.0  # time with two or more batches in flight
    busy: dict = field(default_factory=dict)  # summed per-batch components (s)

    @property
    def qps(self) -> float:
        return self.requests / self.wall_s if self.wall_s > 0 else 0.0

    def summary(self) -> dict:
        lat = self.latencies_s * 1e3
        return {"rate_per_s": self.rate, "requests": self.requests, "queries_per_s": self.qps,
                "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                "mean_ms": float(lat.mean()), "max_ms": float(lat.max()), "batches": self.batches,
                "mean_batch": float(np.mean(self.batch_sizes)) if self.batch_sizes else 0.0,
                "overflow_reruns": self.overflowed, "peak_reserved_gb": self.peak_reserved_bytes / 1e9,
                "overlap_s": self.overlap_s, "wall_s": self.wall_s, "busy_s": self.busy}


class Server:
    """Continuous-batching server for mixed queries over `tables`."""

    def __init__(self, tables: B.MixTables, sizer: B.Sizer, plain: Optional[B.PlainRunner] = None,
                 workers: int = 2, max_batch: int = 512, hbm_budget: float = 150e9, margin: float = 1.5,
                 tuning: Optional[dict] = None):
        import torch
        self.tables, self.max_batch = tables, max_batch
        self.budget = int(hbm_budget) - tables.bytes()
        if self.budget <= 0:
            raise ValueError("the resident tables alone exceed the HBM budget")
        self.device = torch.cuda.current_device()
        self.runners = [B.BatchRunner(tables, sizing="learned", sizer=sizer, plain=plain, margin=margin,
                                      use_graph=False, tuning=tuning) for _ in range(workers)]

    def close(self) -> None:
        for r in self.runners:
            r.close()

    def serve(self, trace: Sequence[Request], on_result=None) -> tuple:
        """Replay `trace` in real time; returns (results by request id,
        report). With `on_result(id, result)` each answer is handed over as
        it completes (from the worker thread, as a view of the pinned buffer
        it arrived in) and not kept; otherwise answers are copied out."""
        import torch
        n = len(trace)
        results: List[Optional[tuple]] = [None] * n
        done_at = np.zeros(n)
        cv = threading.Condition()
        state = {"next": 0, "arrived": 0, "completed": 0, "reserved": 0, "peak": 0, "inflight": 0,
                 "overlap": 0.0, "mark": None, "batches": [], "overflowed": 0, "error": None,
                 "busy": {"batch_wall": 0.0, "execute": 0.0, "features": 0.0, "predict": 0.0, "collect": 0.0,
                          "plan": 0.0, "unpack": 0.0, "fallback": 0.0}}
        cost = [query_hbm_bytes(r.query, self.tables.dim_max_key) for r in trace]
        t0 = time.perf_counter()

        def admit():
            # requests that have arrived, in arrival order, while they fit the budget
            take = []
            i = state["next"]
            free = self.budget - state["reserved"]
            while i < state["arrived"] and len(take) < self.max_batch and cost[i] <= free:
                take.append(i)
                free -= cost[i]
                i += 1
            if not take and i < state["arrived"] and state["reserved"] == 0:
                state["error"] = MemoryError(f"request {i} needs {cost[i]} B, more than the HBM budget")
            return take

        def worker(runner: B.BatchRunner):
            torch.cuda.set_device(self.device)
            while True:
                with cv:
                    while True:
                        if state["error"] is not None or state["next"] >= n:
                            return
                        take = admit()
                        if take:
                            break
                        if state["error"] is not None:
                            cv.notify_all()
                            return
                        cv.wait(timeout=0.05)
                    state["next"] = take[-1] + 1
                    bytes_ = sum(cost[i] for i in take)
                    state["reserved"] += bytes_
                    state["peak"] = max(state["peak"], state["reserved"])
                    now = time.perf_counter()
                    if state["inflight"] >= 1 and state["mark"] is None:
                        state["mark"] = now
                    state["inflight"] += 1
                try:
                    # kept answers leave the pinned buffer at once, so it returns
                    # to the pool however long callers keep them
                    res, rep = runner.run([trace[i].query for i in take], copy=on_result is None)
                except Exception as e:  # surfaced to the caller
                    with cv:
                        state["error"] = e
                        cv.notify_all()
                    return
                t_done = time.perf_counter() - t0
                if on_result is not None:
                    for j, i in enumerate(take):
                        on_result(i, res[j])
                    res = [None] * len(take)
                with cv:
                    for j, i in enumerate(take):
                        results[i] = res[j]
                        done_at[i] = t_done
                    state["completed"] += len(take)
                    state["reserved"] -= bytes_
                    state["batches"].append(len(take))
                    state["overflowed"] += len(rep.overflowed)
                    bz = state["busy"]
                    bz["batch_wall"] += rep.wall_s
                    bz["execute"] += rep.execute_ms / 1e3
                    bz["features"] += rep.features_ms / 1e3
                    bz["predict"] += rep.predict_ms / 1e3
                    bz["collect"] += rep.collect_ms / 1e3
                    bz["plan"] += rep.plan_ms / 1e3
                    bz["unpack"] += rep.unpack_ms / 1e3
                    bz["fallback"] += rep.fallback_s
                    state["inflight"] -= 1
                    if state["inflight"] < 2 and state["mark"] is not None:
                        state["overlap"] += time.perf_counter() - state["mark"]
                        state["mark"] = None
                    cv.notify_all()

        threads = [threading.Thread(target=worker, args=(r,), daemon=True) for r in self.runners]
        for th in threads:
            th.start()
        # release requests at their arrival times
        for k, r in enumerate(trace):
            if state["error"] is not None:
                break
            delay = r.arrival - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            with cv:
                state["arrived"] = k + 1
                cv.notify_all()
        for th in threads:
            th.join()
        if state["error"] is not None:
            raise state["error"]
        wall = float(done_at.max()) if n else 0.0
        lat = done_at - np.array([r.arrival for r in trace])
        rate = n / trace[-1].arrival if n and trace[-1].arrival > 0 else 0.0
        rep = ServeReport(rate=rate, requests=n, wall_s=wall, latencies_s=lat, batches=len(state["batches"]),
                          batch_sizes=state["batches"], overflowed=state["overflowed"],
                          peak_reserved_bytes=state["peak"], overlap_s=state["overlap"], busy=state["busy"])
        return results, rep


def serve_plain_live(plain: B.PlainRunner, trace: Sequence[Request]):
    """The one-query-at-a-time baseline, live: one server thread replays
    `trace` in real time, each request waiting for its arrival and for the
    request before it, then running alone through the plain engine path.
    Latency = completion - arrival on the host clock."""
    import torch
    n = len(trace)
    results, done = [], np.zeros(n)
    t0 = time.perf_counter()
    for k, r in enumerate(trace):
        wait = r.arrival - (time.perf_counter() - t0)
        if wait > 0:
            time.sleep(wait)
        results.append(plain.run(r.query))
        if torch.cuda.is_available():
            torch.cuda.synchronize()
        done[k] = time.perf_counter() - t0
    lat = done - np.array([r.arrival for r in trace])
    rate = n / trace[-1].arrival if n and trace[-1].arrival > 0 else 0.0
    rep = ServeReport(rate=rate, requests=n, wall_s=float(done.max()) if n else 0.0, latencies_s=lat,
                      batches=n, batch_sizes=[1] * n)
    return results, rep


def serve_plain(plain: B.PlainRunner, trace: Sequence[Request], service_s: Optional[np.ndarray] = None):
    """The one-query-at-a-time baseline: every request runs alone through
    the plain engine path, in arrival order behind one FIFO queue. Service
    times are measured by running each query for real; completion times
    follow the queue (completion = max(arrival, previous completion) +
    service), which is exactly what a single server that never overlaps
    requests produces."""
    import torch
    results = []
    if service_s is None:
        service_s = np.zeros(len(trace))
        for k, r in enumerate(trace):
            t = time.perf_counter()
            results.append(plain.run(r.query))
            torch.cuda.synchronize()
            service_s[k] = time.perf_counter() - t
    done = np.zeros(len(trace))
    prev = 0.0
    for k, r in enumerate(trace):
        prev = max(r.arrival, prev) + service_s[k]
        done[k] = prev
    lat = done - np.array([r.arrival for r in trace])
    rate = len(trace) / trace[-1].arrival if trace and trace[-1].arrival > 0 else 0.0
    rep = ServeReport(rate=rate, requests=len(trace), wall_s=float(done.max()) if len(trace) else 0.0,
                      latencies_s=lat, batches=len(trace), batch_sizes=[1] * len(trace))
    return results, rep, service_s
