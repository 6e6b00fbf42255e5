"""Autotuner for the generated kernels and the batched path.

Picks, per plan template and per table-size bucket on the current device,
the tuning the runtime compiler and the batch kernels take: block size,
rows per tile (items per thread = tile rows / consumer threads), TMA ring
depth, occupancy hint, hash-table layout (linear probing / 8-slot buckets)
and shared-memory pre-aggregation versus global atomics (smem=0). Search is
coordinate descent from the default: each parameter in turn is swept with
the others held at the best so far, for `rounds` passes. Every candidate's
result must equal the default tuning's result exactly before its time
counts, so tuning never changes an answer. Winners persist in a JSON cache
(one file per device name) that `Context.prepare(spec, tune="auto")` and
`bench.py --tune auto` read.

The reference has no tuner: its block sizes and strategies are fixed in
the plan builder (metal_plan_builder.cpp) and the executor
(metal_generic_executor.cpp:238-275).
"""
from __future__ import annotations

import json
import math
import os
import time
from pathlib import Path
from typing import Callable, Dict, List, Optional, Sequence, Tuple

CACHE_DIR = Path(os.environ.get("GPUDB_TUNE_DIR", Path(__file__).resolve().parent / "_tune"))

# parameter -> values tried, per template family (first value = default)
SCAN_SPACE = {
    "bs": ["512", "256", "1024"],
    "tile": ["0", "512", "1024", "2048", "4096"],
    "stages": ["4", "2", "3", "6"],
    "occ": ["1", "2", "3", "4", "8"],
}
HASH_SPACE = {
    "layout": ["linear", "bucket8", "packed"],
    "smem": ["10", "0", "8", "12"],
    "sprobe": ["0", "4", "2"],
    "warp": ["1", "0"],
}
SPACES = {
    "q1": {**SCAN_SPACE, "keyed": ["0", "1", "2", "3", "4", "5"], "vec": ["0", "2", "4"], "l2pf": ["0", "1", "2"]},
    "q6": {**SCAN_SPACE, "l2pf": ["0", "1", "2"], "vec": ["0", "2"]},
    "join_topk": {**SCAN_SPACE, "warp": ["1", "0"], "split": ["1", "0"], "bbs": ["0", "256"], "bvec": ["0", "4"]},
    "groupby": {**SCAN_SPACE, **HASH_SPACE},
    "hashjoin": {**SCAN_SPACE, "layout": ["linear", "bucket8"], "probe": ["128", "64", "256"],
                 "smem": ["10", "0", "8"], "warp": ["1", "0"], "sprobe": ["0", "4", "1"], "vec": ["0", "2", "4"]},
}
# Joint moves coordinate descent cannot make one parameter at a time (a
# shallower TMA ring frees the shared memory that a higher occupancy needs):
# measured alongside the default before the descent starts from the best.
SEEDS = {
    # thread-private shared-memory accumulators need a small ring next to
    # their slots for two CTAs per SM: 512-row tiles, two stages
    # ... and with a two-stage ring the L2 prefetch of the next round of
    # tiles keeps DRAM busy (measured 41 us against 44 us without)
    "q1": [{"keyed": "5", "bs": "256", "tile": "448", "stages": "2", "occ": "2", "vec": "2", "l2pf": "1"},
           {"keyed": "5", "bs": "256", "tile": "512", "stages": "2", "occ": "2", "vec": "2"},
           {"keyed": "5", "bs": "256", "tile": "448", "stages": "2", "occ": "2", "vec": "2"},
           {"bs": "256", "stages": "2", "occ": "2"}, {"tile": "2048"}],
    "q6": [{"stages": "2"}, {"bs": "256", "stages": "2", "occ": "2"}, {"stages": "2", "l2pf": "1"},
           {"bs": "256", "stages": "2", "occ": "2", "l2pf": "1"}],
    "join_topk": [{"split": "0", "stages": "2", "warp": "0"}, {"split": "1", "stages": "2"}, {"split": "1", "stages": "2", "occ": "3"},
                  {"split": "1", "stages": "2", "occ": "4", "warp": "0"},
                  {"split": "1", "stages": "2", "occ": "4", "warp": "0", "bvec": "4"}],
    "groupby": [{"bs": "256", "stages": "2", "smem": "8", "warp": "0"},
                {"bs": "256", "stages": "2", "smem": "8", "warp": "0", "layout": "packed"},
                {"bs": "256", "stages": "2", "smem": "8", "warp": "0", "sprobe": "4"}],
    # ... and the probe's latency-bound table lookups gain from every
    # thread slot resident (256-thread CTAs, 512-row tiles, 8 per SM):
    # 1.93 ms against 2.14 ms per step; reading the staged rows four at a
    # time: 1.84 ms
    "hashjoin": [{"stages": "2"}, {"smem": "0", "warp": "1"}, {"stages": "2", "smem": "8", "warp": "0"},
                 {"bs": "256", "stages": "2", "smem": "8", "warp": "0", "occ": "8", "tile": "512"},
                 {"bs": "256", "stages": "2", "smem": "8", "warp": "0", "occ": "8", "tile": "512", "vec": "4"}],
}
BATCH_SPACE = {
    "block": [512, 256, 1024],
    "tile_rows": [32768, 16384, 65536, 4096],
    "warp_aggregate": [True, False],
    "group_rows": [1, 2, 4],
    "agg_rows": [2, 4],
}


def device_key() -> str:
    try:
        import torch
        if torch.cuda.is_available():
            return torch.cuda.get_device_name(0).replace(" ", "_")
    except Exception:
        pass
    return "unknown"


def size_bucket(rows: int) -> str:
    """Tables within a factor of 4 share a tuning."""
    return f"r{int(math.log(max(rows, 1), 4))}"


class TuneCache:
    def __init__(self, path: Optional[Path] = None):
        self.path = Path(path) if path else CACHE_DIR / f"{device_key()}.json"
        self.data: Dict[str, dict] = {}
        if self.path.exists():
            try:
                self.data = json.loads(self.path.read_text())
            except (OSError, ValueError):
                self.data = {}

    @staticmethod
    def key(template: str, rows: int) -> str:
        return f"{template}/{size_bucket(rows)}"

    def get(self, template: str, rows: int) -> Optional[str]:
        e = self.data.get(self.key(template, rows))
        return e["tune"] if e else None

    def put(self, template: str, rows: int, tune: str, ms: float, default_ms: float) -> None:
        self.data[self.key(template, rows)] = {"tune": tune, "ms": ms, "default_ms": default_ms,
                                               "when": time.strftime("%Y-%m-%dT%H:%M:%S")}
        # replicas of a multi-GPU run tune at the same time: under an
        # exclusive lock each re-reads the file, merges its own entry into
        # it and renames its own temporary copy over it, so no replica's
        # entry is lost; a cache that cannot be written only costs a
        # re-tune later
        tmp = self.path.with_suffix(f".{os.getpid()}.tmp")
        try:
            self.path.parent.mkdir(parents=True, exist_ok=True)
            with open(self.path.with_suffix(".lock"), "a") as lk:
                try:
                    import fcntl
                    fcntl.flock(lk.fileno(), fcntl.LOCK_EX)
                except (ImportError, OSError):
                    pass
                try:
                    merged = json.loads(self.path.read_text()) if self.path.exists() else {}
                    if not isinstance(merged, dict):
                        merged = {}
                except (OSError, ValueError):
                    merged = {}
                merged[self.key(template, rows)] = self.data[self.key(template, rows)]
                for k, v in merged.items():
                    self.data.setdefault(k, v)
                tmp.write_text(json.dumps(merged, indent=1, sort_keys=True))
                tmp.replace(self.path)
        except OSError:
            try:
                tmp.unlink()
            except OSError:
                pass


def _tune_string(cfg: Dict[str, str]) -> str:
    return ";".join(f"{k}={v}" for k, v in cfg.items())


def coordinate_descent(space: Dict[str, Sequence], measure: Callable[[dict], Optional[float]],
                       rounds: int = 2, log: Optional[List[dict]] = None,
                       seeds: Sequence[dict] = ()) -> Tuple[dict, float, float]:
    """Minimise measure(cfg) over `space` one parameter at a time, starting
    from the best of the default and the `seeds` (partial configurations
    over the default). measure returns None for a candidate that is
    invalid (fails to build, or its result differs from the default's).
    Returns (best cfg, its time, the default's time)."""
    best = {k: v[0] for k, v in space.items()}
    best_t = measure(best)
    if best_t is None:
        raise RuntimeError("the default tuning does not run")
    default_t = best_t
    seen = {tuple(sorted(best.items())): best_t}
    for seed in seeds:
        cand = {**best, **{k: v for k, v in seed.items() if k in space}}
        sig = tuple(sorted(cand.items()))
        if sig in seen:
            continue
        t = measure(cand)
        seen[sig] = t
        if log is not None:
            log.append({"cfg": cand, "ms": t})
        if t is not None and t < best_t * 0.98:
            best, best_t = cand, t
    for _ in range(rounds):
        improved = False
        for k, values in space.items():
            for v in values:
                cand = dict(best)
                cand[k] = v
                sig = tuple(sorted(cand.items()))
                if sig in seen:
                    t = seen[sig]
                else:
                    t = measure(cand)
                    seen[sig] = t
                    if log is not None:
                        log.append({"cfg": cand, "ms": t})
                if t is not None and t < best_t * 0.98:  # a 2 % margin against noise
                    best, best_t, improved = cand, t, True
        if not improved:
            break
    return best, best_t, default_t


def tune_query(ctx, spec: str, rows: int, template: Optional[str] = None, space: Optional[dict] = None,
               reps: int = 10, warmup: int = 3, rounds: int = 2, cache: Optional[TuneCache] = None,
               log: Optional[List[dict]] = None, flush: Optional[Callable[[], None]] = None,
               timer: Optional[Callable[[object], float]] = None) -> Tuple[str, float, float]:
    """Tune one plan on the tables registered in `ctx`; returns (tune
    string, best ms, default ms) and stores the winner in `cache`. With
    `flush` (which must order its work before the context's next run, e.g.
    on the context's stream), it runs before every timed repetition: inputs
    that L2 could partly hold are then timed from DRAM, as in the bench.
    With `timer(query) -> ms`, each candidate whose answer matched is timed
    by it instead: the caller's own regime (e.g. back-to-back launches over
    rotated input copies), whose ranking of candidates can differ from
    single launches'."""
    from .engine import GpudbError

    template = template or dict(kv.split("=", 1) for kv in spec.split(";") if "=" in kv).get("template", spec)
    space = space or SPACES.get(template, SCAN_SPACE)
    ref = {}

    def canon(res):
        return (tuple(res.types), tuple(tuple(r) for r in res.rows))

    def measure(cfg: dict) -> Optional[float]:
        tune = _tune_string(cfg)
        try:
            q = ctx.prepare(spec, tune)
            res, _ = ctx.run(q)
            if "r" not in ref:
                ref["r"] = canon(res)
            elif canon(res) != ref["r"]:
                return None  # a tuning may never change an answer
            if timer is not None:
                return timer(q)
            for _ in range(warmup):
                ctx.run(q, collect=False)
            ts = []
            for _ in range(reps):
                if flush is not None:
                    flush()
                _, t = ctx.run(q, collect=False)
                ts.append(sum(t.phase_ms))
            ts.sort()
            return ts[len(ts) // 2]
        except (GpudbError, RuntimeError, ValueError):
            return None

    # bring the GPU to its working clocks before anything is compared
    q0 = ctx.prepare(spec, _tune_string({k: v[0] for k, v in space.items()}))
    t_end = time.perf_counter() + 0.5
    while time.perf_counter() < t_end:
        ctx.run(q0, collect=False)
    best, best_t, default_t = coordinate_descent(space, measure, rounds=rounds, log=log,
                                                 seeds=SEEDS.get(template, ()))
    tune = _tune_string(best)
    if cache is not None:
        cache.put(template, rows, tune, best_t, default_t)
    return tune, best_t, default_t


def tune_batch(runner_factory: Callable[[dict], object], queries, space: Optional[dict] = None, reps: int = 3,
               rounds: int = 1, log: Optional[List[dict]] = None) -> Tuple[dict, float, float]:
    """Tune the batch kernels (block size, rows per work item, warp
    aggregation) for a set of queries. runner_factory(tuning) returns a
    BatchRunner; its results must equal the default tuning's."""
    from . import batch as B
    space = space or BATCH_SPACE
    ref = {}

    def measure(cfg: dict) -> Optional[float]:
        r = runner_factory(cfg)
        try:
            res, _ = r.run(queries)
            if "r" not in ref:
                ref["r"] = res
            elif not all(B.same_result(a, b) for a, b in zip(res, ref["r"])):
                return None
            ts = []
            for _ in range(reps):
                _, rep = r.run(queries)
                ts.append(rep.execute_ms)
            return min(ts)
        finally:
            r.close()

    return coordinate_descent(space, measure, rounds=rounds, log=log)


def measure_agg_modes(tables, rows: int, cards=(16, 256, 1024, 8192, 65536, 524288, 4194304),
                      keys=("m_rank_u", "m_rank_z"), thr: int = 5000, reps: int = 3,
                      tuning: Optional[dict] = None) -> List[dict]:
    """Device time of the batched group-by stage for one query of `rows`
    rows per aggregation strategy, over key cardinalities and key skew
    (uniform m_rank_u / Zipf m_rank_z): the measurements behind the
    strategy policy of the batched path."""
    from . import batch as B
    out = []
    for key in keys:
        for card in cards:
            q = B.MixQuery("groupby", 0, 0, rows, thr, key=key, card=card)
            row = {"key": key, "card": card}
            modes = ((B.AGG_SHARED, "shared"), (B.AGG_GLOBAL_WARP, "global_warp"), (B.AGG_GLOBAL, "global"))
            if card <= B.DIRECT_MAX_CARD:
                modes += ((B.AGG_SHARED_DIRECT, "direct"),)
            for mode, name in modes:
                b = B.Batch()
                try:
                    if tuning:
                        b.set_tuning(**tuning)
                    b.set_queries([tables.query_struct(q)])
                    _, d, _ = b.exact_stats()
                    b.set_groups(0, max(1, int(d[0])))
                    b.set_agg_mode(0, mode)
                    ts = []
                    for _ in range(reps + 1):
                        b.execute(use_graph=False)
                        ts.append(b.stage_ms()["group"])
                    row[name + "_ms"] = min(ts[1:])
                    row["groups"] = int(d[0])
                finally:
                    b.close()
            out.append(row)
    return out
