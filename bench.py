"""Benchmark of the runtime-codegen hot path on one B200.

Default workload (the join configuration of the benchmark set): build side
15M rows (unique int32 keys from a seeded permutation, order_day, segment),
probe side 60M rows (fk, ship_day, price, discount); build filter segment==1
AND order_day<1170, probe filter ship_day>1170, group by build key summing
price*(100-discount) exactly in int64, top 10 by (sum desc, key asc).
One step = one full query of five kernels with no host round trip: bitmap
semi-join build; probe listing the matched rows and popcounting the bitmap's
keys; initialisation of the group table sized on the device from those two
counters; gather + hash group-by of the listed rows; top-k.
Seeded synthetic data of the configuration's shapes; inputs exceed the
126 MB L2, so no flush is needed between steps.

Other workloads (`--workload`, for profiling and per-configuration numbers):
q1 (6,001,215-row scan-filter-group-aggregate), q6 (predicate variant),
groupby (120M Zipf(1.1) keys over 2^22, count+sum), hashjoin (2^22-key
build, 120M-row probe, per-key sums).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload W]

Under torchrun every rank runs an independent replica on its own GPU
(replicas only: the query does not shard); the timed region is bracketed by
a barrier and the slowest rank's time is reported.
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import statistics
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """SM clock and clock-event reasons sampled through NVML every ~2 ms
    during the timed region (reads only; no GPU setting is changed)."""

    REASONS = {"hw_slowdown": "nvmlClocksEventReasonHwSlowdown",
               "hw_thermal_slowdown": "nvmlClocksEventReasonHwThermalSlowdown",
               "sw_thermal_slowdown": "nvmlClocksEventReasonSwThermalSlowdown",
               "sw_power_cap": "nvmlClocksEventReasonSwPowerCap"}

    def __init__(self, device: int):
        vis = [v.strip() for v in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if v.strip()]
        self.sel = vis[device] if device < len(vis) else str(device)
        self.samples = []
        self.smax = None
        self.stop = threading.Event()
        self.nv = None

    def __enter__(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            self.nv = nv
            self.h = (nv.nvmlDeviceGetHandleByUUID(self.sel) if self.sel.startswith(("GPU-", "MIG-"))
                      else nv.nvmlDeviceGetHandleByIndex(int(self.sel)))
            self.smax = nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM)
            self._sample()  # one sample at each end of the region, others every ~2 ms
            self.thread = threading.Thread(target=self._run, daemon=True)
            self.thread.start()
        except Exception:
            self.nv = None
        return self

    def _sample(self):
        nv = self.nv
        try:
            self.samples.append((nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM),
                                 nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)))
        except Exception:
            pass

    def _run(self):
        while not self.stop.is_set():
            self._sample()
            time.sleep(0.002)

    def __exit__(self, *a):
        self.stop.set()
        if self.nv:
            self.thread.join(timeout=2)
            self._sample()
            try:
                self.nv.nvmlShutdown()
            except Exception:
                pass

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.smax, "reasons": [], "samples": 0}
        bits = 0
        for _, r in self.samples:
            bits |= r
        reasons = [n for n, attr in self.REASONS.items() if bits & getattr(self.nv, attr, 0)]
        return {"sm_mhz": statistics.median(c for c, _ in self.samples), "sm_max_mhz": self.smax,
                "reasons": reasons, "samples": len(self.samples)}


def dist_info():
    from gpudbmetalcodegen_b200 import replicas
    return replicas.dist_info()


# ---------------------------------------------------------------------------
# workloads
# ---------------------------------------------------------------------------
class Workload:
    name = ""
    spec = ""
    kernel = ""           # dominant kernel (roofline)
    description = ""

    def __init__(self, args):
        self.args = args

    def generate(self):
        raise NotImplementedError

    def rows(self) -> int:
        raise NotImplementedError

    def register(self, ctx):
        for tname, table in self.tables.items():
            ctx.upload_table(tname, table)

    def algorithmic_bytes(self, tune: str) -> dict:
        raise NotImplementedError

    def expected(self):
        raise NotImplementedError

    def matches(self, res) -> bool:
        return res.rows == self.expected()

    def cpu_run(self, threads: int):
        raise NotImplementedError

    def late_columns(self, tune) -> set:
        """(table, column) pairs the plan materialises late."""
        return set()

    def input_bytes(self) -> int:
        """Bytes of every resident column the plan may read."""
        return sum(a.nbytes for t in self.tables.values() for a in t.values())

    def flush_l2(self) -> bool:
        # inputs under twice the L2 could partly survive in it from one
        # timed step to the next: a 256 MB write between steps evicts them
        return self.input_bytes() < 2 * L2_BYTES

    # the table the end-to-end run streams from host memory in chunks, and
    # the tuning of the plan it streams (None: no streamed form)
    stream_table = None

    def stream_tune(self, tune: str):
        return None

    def config(self) -> dict:
        return {"workload": self.description}


class JoinTopK(Workload):
    name = "join_topk"
    kernel = "JT_probe_group"

    def __init__(self, args):
        super().__init__(args)
        self.build_rows, self.probe_rows, self.k = args.build_rows, args.probe_rows, 10
        self.spec = f"template=join_topk;k={self.k}"
        self.description = f"join_topk: build {self.build_rows} + probe {self.probe_rows} rows, top-{self.k}"

    def generate(self):
        from gpudbmetalcodegen_b200 import workloads as W
        self.tables = {"dim": W.gen_dim(self.build_rows, seed=W.SEED),
                       "probe": W.gen_probe(self.probe_rows, dim_rows=self.build_rows, seed=W.SEED)}

    def rows(self):
        return self.build_rows + self.probe_rows

    def expected(self):
        if not hasattr(self, "_exp"):
            from oracle import oracle_py as O
            self._exp, self.groups, self.distinct = O.join_topk(self.tables["dim"], self.tables["probe"], k=self.k)
        return self._exp

    def kernel_for(self, tune):
        # the split plan (the default) only lists matched rows in the probe;
        # JT_group aggregates them. split=0 probes and groups in one kernel
        return "JT_probe_group" if "split=0" in tune else "JT_probe"

    def algorithmic_bytes(self, tune):
        # eager columns (fk, ship_day) for every probe row + the late
        # price/discount (8 B each) for rows reaching the aggregation; with
        # in the split plan the dominant kernel (JT_probe) reads the eager columns only
        import numpy as np
        dim, probe = self.tables["dim"], self.tables["probe"]
        qual = np.zeros(self.build_rows + 2, dtype=bool)
        keep = (dim["b_segment"] == 1) & (dim["b_order_day"] < 1170)
        qual[dim["b_key"][keep]] = True
        passing = probe["p_ship_day"] > 1170
        matched = int(np.count_nonzero(passing & qual[probe["p_fk"]]))
        self.bitmap_lookups = int(np.count_nonzero(passing))
        late = "late=0" not in tune
        alg = self.probe_rows * 8 + matched * 16 if late else self.probe_rows * 24
        if "split=0" not in tune:
            alg = self.probe_rows * 8
        return {"algorithmic_bytes": alg, "rows_reaching_aggregation": matched,
                "all_columns_bytes": self.probe_rows * 24,
                # every column the query references, each read once (build
                # 9 B/row, probe 24 B/row), whatever late materialisation skips
                "query_bytes": self.build_rows * 9 + self.probe_rows * 24}

    def limiter(self, tune, kernel_ms, sm_mhz):
        """The split probe's bound: each row passing the ship-day filter
        looks up a random word of a bitmap far larger than L1, one L2 sector
        request, at about one request per SM clock."""
        if "split=0" in tune or not kernel_ms or not sm_mhz:
            return {}
        floor_ms = self.bitmap_lookups / (148 * sm_mhz * 1e6) * 1e3
        return {"limiter": "l1_miss_requests", "bitmap_lookups": self.bitmap_lookups,
                "request_floor_ms": floor_ms, "request_frac": floor_ms / kernel_ms}

    def cpu_run(self, threads):
        from oracle import oracle_py as O
        O.join_topk(self.tables["dim"], self.tables["probe"], k=self.k, threads=threads)

    def late_columns(self, tune):
        # read only by probe rows that pass the filter and the semi-join
        return set() if "late=0" in tune else {("probe", "p_price"), ("probe", "p_discount")}

    stream_table = "probe"

    def stream_tune(self, tune):
        # the split plan's group phase reads the probe table after the
        # probe, so the streamed form is the unsplit plan of the same tuning
        kv = [t for t in tune.split(";") if t and not t.startswith("split=")]
        return ";".join(kv + ["split=0"])

    def config(self):
        self.expected()
        return {"workload": self.description, "build_rows": self.build_rows, "probe_rows": self.probe_rows,
                "k": self.k, "groups": self.groups, "build_distinct": self.distinct}


class FactScan(Workload):
    def __init__(self, args, which):
        super().__init__(args)
        self.which = which
        self.n = args.fact_rows
        self.spec = f"template={which}"
        self.kernel = {"q1": "Q1_reduce", "q6": "Q6_reduce", "q6_selvec": "Q6S_select"}[which]
        # one scan phase accumulating into zero-filled aggregates: streamable
        # (the selection-vector form's bitmap is indexed by chunk rows: not)
        self.stream_table = "fact" if which in ("q1", "q6") else None
        self.description = {
            "q1": f"q1: scan-filter-group-aggregate over {self.n} rows x 38 B",
            "q6": f"q6: scan-filter-sum over {self.n} rows x 28 B",
            "q6_selvec": f"q6_selvec: the q6 predicate into a selection bitmap (20 B/row), then the sum over the "
                         f"selected rows of {self.n}"}[which]

    def generate(self):
        from gpudbmetalcodegen_b200 import workloads as W
        self.tables = {"fact": W.gen_fact(self.n)}

    def rows(self):
        return self.n

    def stream_tune(self, tune):
        return tune if self.stream_table else None

    def expected(self):
        from oracle import oracle_py as O
        f = self.tables["fact"]
        if self.which != "q1":
            return [(O.q6(f),)]
        return O.q1(f)

    def matches(self, res):
        exp = self.expected()
        if self.which != "q1":
            return res.rows == exp
        got = res.as_dicts()
        from oracle import oracle_py as O
        return len(got) == len(exp) and all(g[k] == e[k] for g, e in zip(got, exp) for k in O.Q1_AGGS)

    def algorithmic_bytes(self, tune):
        # every referenced column once at its declared width; the selection
        # bitmap plan's dominant (first) kernel reads the predicate's three
        # columns, 20 B/row
        per_row = {"q1": 38, "q6": 28, "q6_selvec": 20}[self.which]
        return {"algorithmic_bytes": self.n * per_row, "query_bytes": self.n * (38 if self.which == "q1" else 28)}

    def cpu_run(self, threads):
        from oracle import oracle_py as O
        (O.q1 if self.which == "q1" else O.q6)(self.tables["fact"], threads=threads)


class Skew(Workload):
    def __init__(self, args, which):
        super().__init__(args)
        self.which = which
        self.n = args.zprobe_rows
        self.nkeys = args.zkeys
        self.spec = f"template={which}"
        self.kernel = "GB_aggregate" if which == "groupby" else "HJ_probe_count"
        self.description = (f"{which}: {self.n} probe rows, Zipf(1.1) keys over {self.nkeys}")

    def generate(self):
        from gpudbmetalcodegen_b200 import workloads as W
        self.tables = {"zprobe": W.gen_zprobe(self.n, nkeys=self.nkeys)}
        if self.which == "hashjoin":
            self.tables["zbuild"] = W.gen_zbuild(self.nkeys)

    def register(self, ctx):
        super().register(ctx)
        ctx.register_symbol("zgroups", self.nkeys)

    def rows(self):
        return self.n + (self.nkeys if self.which == "hashjoin" else 0)

    def expected(self):
        from oracle import oracle_py as O
        zp = self.tables["zprobe"]
        if self.which == "groupby":
            return O.groupby(zp["z_key"], zp["z_value"], cap=self.nkeys)
        return O.hashjoin(self.tables["zbuild"], zp["z_key"], cap=self.nkeys)

    def matches(self, res):
        import numpy as np
        k, c, s = self.expected()
        return (np.array_equal(np.array(res.column("key")), k) and np.array_equal(np.array(res.column("count")), c)
                and np.array_equal(np.array(res.column("sum")), s))

    def algorithmic_bytes(self, tune):
        return {"algorithmic_bytes": self.n * (16 if self.which == "groupby" else 8)}

    def cpu_run(self, threads):
        self.expected()


def make_workload(args) -> Workload:
    if args.workload == "join_topk":
        return JoinTopK(args)
    if args.workload in ("q1", "q6", "q6_selvec"):
        return FactScan(args, args.workload)
    if args.workload in ("groupby", "hashjoin"):
        return Skew(args, args.workload)
    raise SystemExit(f"unknown workload {args.workload}")


def time_cpu(w: Workload, budget_s: float = 12.0, max_runs: int = 20):
    threads = os.cpu_count() or 1
    w.cpu_run(threads)
    times = []
    t_end = time.perf_counter() + budget_s
    while len(times) < 3 or (time.perf_counter() < t_end and len(times) < max_runs):
        t0 = time.perf_counter()
        w.cpu_run(threads)
        times.append(time.perf_counter() - t0)
    return statistics.median(times), threads, len(times)


L2_BYTES = 126 << 20  # B200 L2 (126 MB)


def workload_config(w: Workload, world: int) -> dict:
    """The `config` object of both arms' lines: the workload and its sizes,
    how L2 is kept out of the timing, and the replica count."""
    cfg = w.config()
    l2 = ("three device copies of the inputs rotated from step to step (each step reads a copy the other two, "
          "over twice the 126 MB L2, evicted); the tuner flushes L2 before each timed run"
          ) if w.flush_l2() else "inputs larger than twice the 126 MB L2; no flush"
    cfg.update({"l2": l2, "parallelism": f"replicas x{world}"})
    return cfg


def run_reference(args, w: Workload):
    """The reference's operator semantics restated on the CPU (the oracle
    port: the reference's own kernels are Metal and cannot run here), on all
    host cores, same workload and metric."""
    w.generate()
    step, threads, n = time_cpu(w, budget_s=max(5.0, 0.5 * args.steps), max_runs=max(3, args.steps))
    value = w.rows() / step
    line = {"metric": "rows_per_s", "value": value, "unit": "rows/s", "n_gpus": args.gpus, "steps": n,
            "warmup": args.warmup, "ms_per_step": step * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int64", "data": "synthetic (seeded)", "impl": "reference",
            "config": workload_config(w, args.gpus),
            "cpu_baseline": {"value": value, "unit": "rows/s", "cores": threads, "kind": "port",
                             "sample": f"full workload ({w.rows()} rows) per step, {n} steps, median"},
            "e2e": {"value": value, "unit": "rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# mixed-query batches with the learned sizer
# ---------------------------------------------------------------------------
def mixed_oracle_seconds(args, queries, budget_s: float, dim_rows=None, zipf=None):
    """The oracle (the reference's operator semantics restated on the CPU,
    all host cores) over the first queries of the batch until `budget_s`
    has passed; slices are regenerated on the host from the same seeds."""
    from gpudbmetalcodegen_b200 import workloads as W
    from oracle import oracle_py as O
    threads = os.cpu_count() or 1
    dim_rows = dim_rows or args.mix_dim_rows
    zipf = zipf or W.MIX_ZIPF_S
    seed = W.SEED if zipf is W.MIX_ZIPF_S else W.SEED + 5
    md = W.gen_mixdim(dim_rows, seed=seed)
    done, spent = 0, 0.0
    for q in queries:
        m = W.gen_mix(q.rows, nranks=W.MIX_NRANKS, s=zipf[q.table], dim_rows=dim_rows,
                      seed=seed + 7919 * q.table, row0=q.row0)
        t0 = time.perf_counter()
        if q.tmpl == "agg":
            O.mix_agg(m, q.thr, threads=threads)
        elif q.tmpl == "join":
            O.mix_join(md, m, q.attr_lt, q.thr, threads=threads)
        else:
            k, c, sm = O.mix_groupby(m, q.key, q.thr, q.card, threads=threads)
            if q.tmpl == "topk":
                O.topk(k, sm, q.k)
        spent += time.perf_counter() - t0
        done += 1
        if spent >= budget_s:
            break
    return done, spent, threads


def mixed_oracle_check(tables, queries, results, n: int = 24) -> dict:
    """The oracle (the reference's operator semantics on the CPU) on a
    seeded subset of the batch that holds every template: each query's
    slice is regenerated on the host from the table's seed and compared
    with the engine's answer bit for bit."""
    import numpy as np
    from gpudbmetalcodegen_b200 import batch as B, workloads as W
    from oracle import oracle_py as O
    rng = np.random.default_rng(2024)
    pick = set(int(i) for i in rng.choice(len(queries), min(n, len(queries)), replace=False))
    for t in B.TEMPLATES:
        pick.update([i for i, q in enumerate(queries) if q.tmpl == t][:1])
    md = W.gen_mixdim(tables.dim_rows, seed=tables.seed)
    bad, t0 = [], time.perf_counter()
    for i in sorted(pick):
        q = queries[i]
        m = W.gen_mix(q.rows, nranks=tables.nranks, s=tables.zipf_s[q.table], dim_rows=tables.dim_rows,
                      seed=tables.table_seed(q.table), row0=q.row0)
        if q.tmpl == "agg":
            e = ("scalar",) + tuple(O.mix_agg(m, q.thr))
        elif q.tmpl == "join":
            e = ("scalar",) + tuple(O.mix_join(md, m, q.attr_lt, q.thr))
        else:
            k, c, sm = O.mix_groupby(m, q.key, q.thr, q.card)
            e = B.canonical_groups(k, c, sm) if q.tmpl == "groupby" else ("topk", tuple(O.topk(k, sm, q.k)))
        if not B.same_result(results[i], e):
            bad.append(i)
    return {"queries": len(pick), "templates": sorted({queries[i].tmpl for i in pick}), "mismatches": bad,
            "ok": not bad, "host_s": time.perf_counter() - t0}


def batch_tuning(args) -> dict:
    """The batch kernels' launch shape from --batch-tune ("block=512;tile_rows=65536"), None for the defaults."""
    if not args.batch_tune:
        return None
    out = {}
    for kv in args.batch_tune.split(";"):
        k, v = kv.split("=")
        out[k.strip()] = int(v)
    return out


def run_mixed(args, pg=None):
    """Config: 256 seeded mixed queries over slices (1M-120M rows) of four
    resident 120M-row mix tables. One step = the whole batch through the
    batched, learned-sizing path (4096-row sample features, MLP prediction,
    persistent work-queue kernels in a CUDA graph, one packed result copy,
    exact re-run of any overflowed table). Beside it: the plain
    one-query-at-a-time path (exact count pass + generated kernels per
    query) and the batched path with the exact count pass."""
    import torch
    from gpudbmetalcodegen_b200 import Context, batch as B, workloads as W

    world, rank, local = dist_info()
    if args.impl == "reference":
        if rank == 0:
            qs = W.gen_mixed_queries(args.mix_queries, seed=W.SEED, table_rows=args.mix_rows)
            done, spent, threads = mixed_oracle_seconds(args, qs, budget_s=max(10.0, 2.0 * args.steps))
            v = done / spent
            return ({
                "metric": "mixed_queries_per_s", "value": v, "unit": "queries/s", "n_gpus": args.gpus,
                "steps": 1, "warmup": 0, "ms_per_step": 1e3 * spent / done * args.mix_queries,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
                "data": "synthetic (seeded)", "impl": "reference",
                "config": {"workload": f"mixed: {args.mix_queries} queries over slices of 120M-row tables"},
                "cpu_baseline": {"value": v, "unit": "queries/s", "cores": threads, "kind": "port",
                                 "sample": f"first {done} of the {args.mix_queries} queries"},
                "e2e": {"value": v, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
        return None

    torch.cuda.set_device(local)
    from gpudbmetalcodegen_b200 import replicas
    own_pg = pg is None
    if own_pg:
        pg = replicas.init("nccl", 300)

    t0 = time.perf_counter()
    tables = B.MixTables(rows=args.mix_rows, zipf_s=W.MIX_ZIPF_S, nranks=W.MIX_NRANKS,
                         dim_rows=args.mix_dim_rows, seed=W.SEED)
    gen_s = time.perf_counter() - t0
    queries = W.gen_mixed_queries(args.mix_queries, seed=W.SEED, table_rows=args.mix_rows)
    total_rows = sum(q.rows for q in queries)
    alg_bytes = sum(B.query_bytes(q, args.mix_dim_rows) for q in queries)

    # the sizer: trained on engine-logged executions of other queries
    t0 = time.perf_counter()
    log = B.ExecutionLog()
    train_q = W.gen_mixed_queries(args.train_executions, seed=W.SEED + 1, table_rows=args.mix_rows)
    log_ms = B.log_executions(tables, train_q, log, batch_size=1024)
    log_s = time.perf_counter() - t0
    sizer, sinfo = B.train_sizer(log, seed=1, epochs=args.sizer_epochs, batch=512, lr=3e-3)
    sinfo.update({"executions": len(log), "log_device_ms": log_ms, "log_s": log_s})

    ctx = Context(local)
    plain = B.PlainRunner(ctx, tables)
    # the setup's objects (the training log, the query lists) move to the
    # collector's permanent generation, so its periodic full passes do not
    # scan them in the middle of a timed region
    gc.collect()
    gc.freeze()
    # plain one-query-at-a-time path (first pass compiles / warms)
    plain_res = [plain.run(q) for q in queries]
    torch.cuda.synchronize()
    peak, peak_kind = peaks()
    # the baseline's best pass (its pass-to-pass spread is reported beside it)
    passes = []
    for _ in range(max(1, args.plain_passes)):
        per_tmpl = {}  # template -> [queries, seconds, algorithmic bytes]
        count_s0, count_n0 = plain.count_s, plain.count_passes
        plain_res = []
        t0 = time.perf_counter()
        for q in queries:
            tq = time.perf_counter()
            plain_res.append(plain.run(q))
            d = per_tmpl.setdefault(q.tmpl, [0, 0.0, 0])
            d[0] += 1
            d[1] += time.perf_counter() - tq
            d[2] += B.query_bytes(q, 0)
        torch.cuda.synchronize()
        count_n = plain.count_passes - count_n0
        passes.append((time.perf_counter() - t0, per_tmpl, (plain.count_s - count_s0) / count_n if count_n else None))
    plain_s, per_tmpl, count_mean = min(passes, key=lambda x: x[0])
    # per template: wall time per query against the HBM time of the bytes it
    # must read (the count pass of a grouped query is part of its time)
    plain_breakdown = {t: {"queries": n, "mean_ms": sec / n * 1e3,
                           "hbm_ms": b / n / (peak * 1e9) * 1e3, "x_hbm": sec / (b / (peak * 1e9))}
                       for t, (n, sec, b) in sorted(per_tmpl.items())}
    plain_breakdown["count_pass_mean_ms"] = count_mean * 1e3 if count_mean is not None else None
    plain_breakdown["pass_s"] = [x[0] for x in passes]

    bt = batch_tuning(args)
    exact = B.BatchRunner(tables, sizing="exact", plain=plain, tuning=bt)
    for _ in range(2):
        exact.run(queries)
    t0 = time.perf_counter()
    for _ in range(3):
        exact_res, exact_rep = exact.run(queries)
    exact_s = (time.perf_counter() - t0) / 3
    exact.close()

    learned = B.BatchRunner(tables, sizing="learned", sizer=sizer, plain=plain, tuning=bt)
    for _ in range(args.warmup):
        res, rep = learned.run(queries)
    stream = torch.cuda.current_stream()
    if pg:
        replicas.barrier(pg)
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    reps = []
    launches = 0
    with ClockSampler(local) as clk:
        ev0.record(stream)
        w0 = time.perf_counter()
        for i in range(args.steps):
            res, rep = learned.run(queries)
            reps.append(rep)
            launches += rep.launches + 2  # + the sample kernel and the predictor
        ev1.record(stream)
        ev1.synchronize()
        wall_ms = (time.perf_counter() - w0) * 1e3 / args.steps
    step_ms = ev0.elapsed_time(ev1) / args.steps
    if pg:
        step_ms, wall_ms = replicas.max_over_ranks(pg, [step_ms, wall_ms], "cuda")
        replicas.barrier(pg)
    verified = all(B.same_result(a, b) for a, b in zip(res, plain_res)) and \
        all(B.same_result(a, b) for a, b in zip(exact_res, plain_res))
    # a seeded subset (every template) against the oracle, on slices
    # regenerated on the host from the tables' seeds
    oracle_check = mixed_oracle_check(tables, queries, res, n=24) if rank == 0 else None

    # per-kernel device times (one execute without a graph) for the roofline
    learned.batch.execute(use_graph=False)
    stages = learned.batch.stage_ms()
    grouped_bytes = sum(B.query_bytes(q, 0) for q in queries if q.grouped)
    scalar_bytes = sum(B.query_bytes(q, 0) for q in queries if not q.grouped)
    dom = max(("group", "agg_probe"), key=lambda k: stages[k])
    dom_bytes = grouped_bytes if dom == "group" else scalar_bytes
    achieved = dom_bytes / (stages[dom] / 1e3) / 1e9 if stages[dom] else None
    roofline = {"bound": "hbm", "kernel": "kGroup" if dom == "group" else "kAgg", "achieved": achieved,
                "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak if achieved else None,
                "kernel_ms": stages[dom], "algorithmic_bytes": dom_bytes, "stage_ms": stages,
                "batch_hbm_frac": alg_bytes / (sum(stages.values()) / 1e3) / 1e9 / peak,
                "traffic": load_traffic("kGroup" if dom == "group" else "kAgg")}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        done, spent, threads = mixed_oracle_seconds(args, queries, budget_s=15.0)
        cpu = {"value": done / spent, "unit": "queries/s", "cores": threads, "kind": "port",
               "sample": f"first {done} of the {len(queries)} queries, slices regenerated on the host"}

    n_q = len(queries) * world
    value = n_q / (step_ms / 1e3)
    if rank == 0:
        desc_bytes = len(queries) * 128
        line = {"metric": "mixed_queries_per_s", "value": value, "unit": "queries/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic (seeded)",
                "config": {"workload": f"mixed: {len(queries)} queries (agg / join / groupby / topk) over slices "
                                       f"of {len(W.MIX_ZIPF_S)} resident {args.mix_rows}-row tables, learned sizing",
                           "queries": len(queries), "rows_scanned_per_step": total_rows,
                           "algorithmic_bytes_per_step": alg_bytes, "table_gen_s": gen_s,
                           "l2": "inputs larger than the 126 MB L2; no flush",
                           "parallelism": f"replicas x{world}"},
                "verified": verified, "verified_vs_oracle": oracle_check, "batch_tuning": bt or "default",
                "plain_per_query": {"queries_per_s": len(queries) / plain_s, "ms_per_batch": plain_s * 1e3,
                                    "count_passes": plain.count_passes, "per_template": plain_breakdown},
                "batched_exact": {"queries_per_s": len(queries) / exact_s, "ms_per_batch": exact_s * 1e3,
                                  "stats_ms": exact_rep.stats_ms, "execute_ms": exact_rep.execute_ms,
                                  "collect_ms": exact_rep.collect_ms, "overflowed": len(exact_rep.overflowed),
                                  "fallback_s": exact_rep.fallback_s},
                "batched_learned": {"queries_per_s": len(queries) / (wall_ms / 1e3), "ms_per_batch": wall_ms,
                                    "execute_ms": statistics.median(r.execute_ms for r in reps),
                                    "features_ms": statistics.median(r.features_ms for r in reps),
                                    "collect_ms": statistics.median(r.collect_ms for r in reps),
                                    "overflowed": len(reps[-1].overflowed),
                                    "fallback_s": statistics.median(r.fallback_s for r in reps),
                                    "table_slots": reps[-1].table_slots},
                "speedup_vs_plain": (len(queries) / (wall_ms / 1e3)) / (len(queries) / plain_s),
                "rows_per_s": total_rows * world / (step_ms / 1e3),
                "sizer": sinfo, "roofline": roofline, "cpu_baseline": cpu,
                "e2e": {"value": n_q / (wall_ms / 1e3), "unit": "queries/s", "h2d_bytes_per_step": desc_bytes,
                        "d2h_bytes_per_step": reps[-1].result_bytes,
                        "note": "wall clock through BatchRunner.run; tables resident in HBM by the workload's "
                                "definition, per-step inputs are the query descriptors"},
                "gpu_launches": launches, "clocks": clk.summary()}
    learned.close()
    sizer.close()
    ctx.close()
    gc.unfreeze()
    if own_pg and pg:
        replicas.shutdown(pg)
    return line if rank == 0 else None


def run_serve(args, pg=None):
    """Config: a 120M-row table and a 30M-row dimension resident in HBM;
    mixed queries (the mixed generator, slices of 1M-120M rows) arriving as
    a Poisson process at each offered rate; the continuous-batching server
    (learned sizing, HBM budget, two workers whose batches overlap) against
    the plain one-query-at-a-time path on the same trace. Every served
    answer is checked against the plain path's answer for the same query."""
    import numpy as np
    import torch
    from gpudbmetalcodegen_b200 import Context, batch as B, serve as S, workloads as W

    world, rank, local = dist_info()
    if args.impl == "reference":
        if rank == 0:
            qs = W.gen_mixed_queries(args.serve_queries, seed=W.SEED + 5, table_rows=args.serve_rows, n_tables=1)
            done, spent, threads = mixed_oracle_seconds(args, qs, budget_s=max(10.0, 2.0 * args.steps),
                                                        dim_rows=args.serve_dim_rows, zipf=(W.ZIPF_S,))
            v = done / spent
            return ({
                "metric": "serve_queries_per_s", "value": v, "unit": "queries/s", "n_gpus": args.gpus, "steps": 1,
                "warmup": 0, "ms_per_step": 1e3 * spent / done, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "int64", "data": "synthetic (seeded)", "impl": "reference",
                "config": {"workload": "serve: mixed queries over a resident 120M-row table, one at a time"},
                "cpu_baseline": {"value": v, "unit": "queries/s", "cores": threads, "kind": "port",
                                 "sample": f"first {done} queries of the trace"},
                "e2e": {"value": v, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
        return None
    torch.cuda.set_device(local)
    tables = B.MixTables(rows=args.serve_rows, zipf_s=(W.ZIPF_S,), nranks=W.MIX_NRANKS,
                         dim_rows=args.serve_dim_rows, seed=W.SEED + 5)
    log = B.ExecutionLog()
    t0 = time.perf_counter()
    B.log_executions(tables, W.gen_mixed_queries(args.train_executions, seed=W.SEED + 6,
                                                 table_rows=args.serve_rows, n_tables=1), log, batch_size=1024)
    sizer, sinfo = B.train_sizer(log, seed=1, epochs=args.sizer_epochs, batch=512, lr=3e-3)
    sinfo["log_s"] = time.perf_counter() - t0
    ctx = Context(local)
    plain = B.PlainRunner(ctx, tables)
    qs = W.gen_mixed_queries(args.serve_queries, seed=W.SEED + 5, table_rows=args.serve_rows, n_tables=1)
    rates = [float(r) for r in args.serve_rates.split(",")]
    # the plain path, each query alone: the first run of a query compiles its
    # kernels (constants are part of the generated source), the second is
    # timed with the kernel cache warm -- the service time of the queue
    n_plain = min(args.serve_plain_queries, len(qs))
    compile_s = []
    for q in qs[:n_plain]:
        t = time.perf_counter()
        plain.run(q)
        torch.cuda.synchronize()
        compile_s.append(time.perf_counter() - t)
    plain_res, _, service = S.serve_plain(plain, S.poisson_trace(qs[:n_plain], rate=rates[0], seed=11))
    plain_fp = [B.result_fingerprint(r) for r in plain_res]
    del plain_res
    # every served answer is also checked against one exact-sized batch of all queries
    ex = B.BatchRunner(tables, sizing="exact", plain=plain)
    exact_res, _ = ex.run(qs)
    exact_fp = [B.result_fingerprint(r) for r in exact_res]
    # the exact batch itself against the oracle on a seeded subset (slices
    # regenerated on the host): the served answers are then checked
    # against it, every one of them
    oracle_check = mixed_oracle_check(tables, qs, exact_res, n=16) if rank == 0 else None
    del exact_res
    ex.close()
    srv = S.Server(tables, sizer, plain=plain, workers=args.serve_workers, hbm_budget=150e9,
                   max_batch=args.serve_max_batch)
    srv.serve(S.poisson_trace(qs, rate=rates[-1], seed=12))  # warm the workers, their arenas and pools
    # the setup's objects out of the collector's periodic full passes (a
    # pass over the training log stalls every serving thread)
    gc.collect()
    gc.freeze()
    per_rate, verified, clocks = [], True, None
    launches = 0
    for rate in rates:
        trace = S.poisson_trace(qs, rate=rate, seed=11)
        # the server copies every answer out of its pinned buffer as it
        # completes (part of serving); they are fingerprinted only after the
        # trace, so the check takes no interpreter time from the workers
        with ClockSampler(local) as clk:
            served, rep = srv.serve(trace)
        fps = [B.result_fingerprint(r) for r in served]
        del served
        clocks = clk.summary()
        ok_alone = fps[:n_plain] == plain_fp
        ok_all = fps == exact_fp
        verified = verified and ok_alone and ok_all
        # the baseline served live, one query at a time, on the same arrivals
        live_res, prep = S.serve_plain_live(plain, trace[:n_plain])
        verified = verified and [B.result_fingerprint(r) for r in live_res] == plain_fp
        del live_res
        launches += 7 * rep.batches
        per_rate.append({"offered_per_s": rate, "ours": rep.summary(),
                         f"plain_one_at_a_time_first_{n_plain}": prep.summary(),
                         "bit_exact_vs_alone": ok_alone, "bit_exact_vs_exact_batch": ok_all})
    srv.close()
    gc.unfreeze()
    top = per_rate[-1]["ours"]
    if rank == 0:
        line = {"metric": "serve_queries_per_s", "value": top["queries_per_s"], "unit": "queries/s",
                "n_gpus": world, "steps": len(rates), "warmup": 1, "ms_per_step": top["wall_s"] * 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
                "data": "synthetic (seeded)",
                "config": {"workload": f"serve: {len(qs)} mixed queries per trace over a resident "
                                       f"{args.serve_rows}-row table + {args.serve_dim_rows}-row dimension, Poisson "
                                       f"arrivals, HBM budget 150 GB, {args.serve_workers} workers, at most "
                                       f"{args.serve_max_batch} queries per batch",
                           "rates": rates, "parallelism": "replicas x1"},
                "verified": verified, "verified_vs_oracle": oracle_check, "per_rate": per_rate,
                "plain_service_ms": {"warm_mean": float(service.mean() * 1e3),
                                     "warm_p50": float(np.median(service) * 1e3),
                                     "first_run_with_compile_mean": float(np.mean(compile_s) * 1e3),
                                     "queries": n_plain},
                "sizer": sinfo,
                "e2e": {"value": top["queries_per_s"], "unit": "queries/s", "h2d_bytes_per_step": 128 * len(qs),
                        "d2h_bytes_per_step": None,
                        "note": "wall clock from first arrival to last answer on the host, at the highest offered rate"},
                "gpu_launches": launches, "clocks": clocks}
    sizer.close()
    ctx.close()
    return line if rank == 0 else None


def run_aggmodes(args):
    """The batched group-by stage per aggregation strategy, cardinality and
    key skew: one 60M-row query at 50 % selectivity each."""
    import torch
    from gpudbmetalcodegen_b200 import autotune, batch as B, workloads as W
    world, rank, local = dist_info()
    if args.impl == "reference":
        if rank == 0:
            return {"impl": "reference", "unavailable": "a measurement of the engine's own aggregation strategies only"}
        return None
    torch.cuda.set_device(local)
    rows = args.agg_rows or args.zprobe_rows // 2
    tables = B.MixTables(rows=rows, zipf_s=(W.ZIPF_S,), nranks=W.MIX_NRANKS, dim_rows=1_000_000, seed=W.SEED)
    kw = {}
    if args.agg_cards:
        kw["cards"] = tuple(int(c) for c in args.agg_cards.split(","))
    if args.agg_keys:
        kw["keys"] = tuple(args.agg_keys.split(","))
    table = autotune.measure_agg_modes(tables, rows, tuning=batch_tuning(args), **kw)
    if rank == 0:
        return ({"metric": "group_stage_ms_per_strategy", "value": None, "unit": "ms", "n_gpus": 1,
                          "steps": 3, "warmup": 1, "higher_is_better": False, "dtype": "int64",
                          "data": "synthetic (seeded)", "config": {"workload": f"aggmodes: {rows} rows, thr 5000"},
                          "table": table})
    return None


def load_traffic(kernel: str):
    p = ROOT / "profiles" / "traffic.json"
    if p.exists():
        try:
            return json.loads(p.read_text()).get(kernel)
        except Exception:
            return None
    return None


def measure(args, w: Workload, pg, world: int, rank: int, local: int):
    """One workload through the engine on this rank's GPU: verified first
    run, timed back-to-back graph replays (max over ranks), per-kernel
    times, roofline, end to end from pinned host buffers, and the CPU
    baseline on rank 0. Returns rank 0's JSON line (None elsewhere)."""
    import ctypes as C
    import numpy as np
    import torch

    from gpudbmetalcodegen_b200 import Context, _lib, replicas

    w.generate()
    ctx = Context(local)
    w.register(ctx)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr)
    flush = w.flush_l2()
    scratch = [torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}") for _ in range(2)] if flush else None

    def flush_l2():
        # a 256 MB write evicts the inputs; a 256 MB read of another buffer
        # then leaves L2 holding clean lines, so the timed step pays no
        # write-back of the flush's dirty lines
        if flush:
            with torch.cuda.stream(stream):
                scratch[0].zero_()
                scratch[1].view(torch.int64).sum()
    rot, bind = None, None
    if flush:
        # inputs under twice the L2: three device copies of every column,
        # rotated from step to step, so each step reads a copy that the
        # other two (at least twice the L2) evicted, launches still back to
        # back (each copy's plan is its own cached graph)
        lib = _lib.load()
        rot, held = [], []
        for _ in range(3):
            binds = []
            for tname, table in w.tables.items():
                for cname, arr in table.items():
                    t = torch.from_numpy(np.ascontiguousarray(arr)).to(f"cuda:{local}")
                    held.append(t)
                    binds.append((tname.encode(), cname.encode(), C.c_void_p(t.data_ptr()), arr.shape[0],
                                  arr.itemsize))
            rot.append(binds)

        def bind(k):
            for tb, cb, ptr, n, e in rot[k]:
                lib.gpudb_register_column(ctx.handle, tb, cb, ptr, n, e)

    def rotated_step_ms(qq, steps: int = 30) -> float:
        # a candidate's step as the timed region below measures it: graph
        # replays back to back over the rotated copies (single flushed
        # launches also time each launch's start-up, and rank tiles
        # differently)
        ctx.set_use_graphs(not args.no_graphs)
        try:
            for i in range(6):
                bind(i % 3)
                ctx.enqueue(qq)
            ctx.sync()
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for i in range(steps):
                bind(i % 3)
                ctx.enqueue(qq)
            b.record(stream)
            b.synchronize()
            ctx.sync()
            return a.elapsed_time(b) / steps
        finally:
            ctx.set_use_graphs(False)

    tuner = None
    tune = args.tune
    if tune == "auto":
        # the autotuner's choice for this template and table size (tuned
        # now, untimed, when the device has none stored)
        from gpudbmetalcodegen_b200 import autotune
        cache = autotune.TuneCache()
        tpl = dict(kv.split("=", 1) for kv in w.spec.split(";")).get("template")
        rows = ctx.largest_table_rows()
        if cache.get(tpl, rows) is None or args.tune_search:
            # no stored choice for this device: the default and the seed
            # tunings are measured (answers checked against the first run),
            # the fastest is stored; the full coordinate descent runs with
            # --tune search
            t0 = time.perf_counter()
            tlog = []
            autotune.tune_query(ctx, w.spec, rows, cache=cache, log=tlog, rounds=0 if not args.tune_search else 2,
                                flush=flush_l2 if flush else None, timer=rotated_step_ms if flush else None)
            tuner = {"tuned_s": time.perf_counter() - t0, "candidates": len(tlog) + 1,
                     "mode": "search" if args.tune_search else "seeds"}
        e = cache.data.get(cache.key(tpl, rows), {})
        tuner = {**(tuner or {}), "chosen": e.get("tune"), "tuned_ms": e.get("ms"), "default_ms": e.get("default_ms")}
        tune = ctx.resolve_tune(w.spec, "auto")
    q = ctx.prepare(w.spec, tune)

    verified = None
    if not args.no_verify:
        res, _ = ctx.run(q)
        verified = w.matches(res)

    # the timed steps are enqueued back to back (no host wait between
    # them), each replaying the plan as a CUDA graph (fills and kernels,
    # captured during the warm-up); device errors are read once after the
    # last step. The kernels' own times come from a second, ungraphed pass
    # with an event around every launch.
    kernels = [ln.split()[2].rstrip(":") for ln in q.plan.splitlines() if ln.strip().startswith("phase ")]
    ctx.set_use_graphs(not args.no_graphs)
    for _ in range(args.warmup):
        ctx.enqueue(q)
    ctx.sync()
    phase_acc, names = {}, []
    if pg:
        replicas.barrier(pg)
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)

    if rot:
        # each copy's launch sequence twice: a graph is captured when its
        # sequence recurs, so all three are captured before the timed steps
        for i in range(max(6, args.warmup)):
            bind(i % 3)
            ctx.enqueue(q)
        ctx.sync()
        torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for i in range(args.steps):
            if rot:
                bind(i % 3)
            ctx.enqueue(q)
        ev1.record(stream)
        ev1.synchronize()
    ctx.sync()
    torch.cuda.synchronize()
    # the answer the last timed replay left in the buffers, against the oracle
    verified_timed = None if args.no_verify else w.matches(ctx.collect(q))
    launches = len(kernels) * args.steps
    step_ms = ev0.elapsed_time(ev1) / args.steps
    ctx.set_use_graphs(False)
    phase_steps = max(5, min(args.steps, 20))
    for _ in range(phase_steps):
        flush_l2()
        torch.cuda.synchronize()
        _, t = ctx.run(q, collect=False)
        for i, ms in enumerate(t.phase_ms):
            phase_acc[i] = phase_acc.get(i, 0.0) + ms
    if pg:
        step_ms = replicas.max_over_ranks(pg, [step_ms], "cuda")[0]
        replicas.barrier(pg)
    rows_total = w.rows() * world
    value = rows_total / (step_ms / 1e3)

    phase_ms = {(kernels[i] if i < len(kernels) else str(i)): v / phase_steps for i, v in phase_acc.items()}
    kernel = w.kernel_for(q.tune) if hasattr(w, "kernel_for") else w.kernel
    kms = phase_ms.get(kernel)
    if rot and len(kernels) == 1:
        # one kernel per step: its average duration over the timed region
        # of back-to-back launches (the per-launch events of the pass above
        # also hold each launch's start-up latency)
        kms = step_ms
    peak, peak_kind = peaks()
    ab = w.algorithmic_bytes(q.tune)
    achieved = ab["algorithmic_bytes"] / (kms / 1e3) / 1e9 if kms else None
    roofline = {"bound": "hbm", "kernel": kernel, "achieved": achieved, "peak": peak, "peak_kind": peak_kind,
                "unit": "GB/s", "frac": (achieved / peak) if achieved else None, "kernel_ms": kms,
                "traffic": load_traffic(kernel), **ab}
    if "query_bytes" in ab:
        # whole query per step against the same peak, bytes counted as above
        qg = ab["query_bytes"] / (step_ms / 1e3) / 1e9
        roofline.update({"query_gbs": qg, "query_frac": qg / peak})
    if hasattr(w, "limiter"):
        roofline.update(w.limiter(q.tune, kms, clk.summary().get("sm_mhz")))

    # end to end through the C-ABI with pinned host buffers, per step: H2D
    # of every column the plan reads for all rows, the late-materialised
    # columns read in place from host memory by the rows that reach them
    # (the reference's zero-copy buffers), the query, D2H of the result
    e2e = None
    if not args.no_e2e:
        lib = _lib.load()
        late = w.late_columns(q.tune)
        pinned, host_bytes, late_bytes = [], 0, 0
        for tname, table in w.tables.items():
            for cname, arr in table.items():
                ptr = lib.gpudb_host_alloc(arr.nbytes)
                np.ctypeslib.as_array((C.c_uint8 * arr.nbytes).from_address(ptr))[:] = arr.view(np.uint8)
                in_place = (tname, cname) in late
                pinned.append((tname, cname, ptr, arr, in_place))
                if in_place:
                    late_bytes += arr.itemsize
                else:
                    host_bytes += arr.nbytes

        def e2e_step():
            for tname, cname, ptr, arr, in_place in pinned:
                fn = lib.gpudb_register_host_column if in_place else lib.gpudb_upload_column
                _lib.check(fn(ctx.handle, tname.encode(), cname.encode(), C.c_void_p(ptr), arr.shape[0], arr.itemsize),
                           ctx.handle)
            r, _ = ctx.run(q, collect=True)
            return r

        for _ in range(2):
            r = e2e_step()
        ctx.synchronize()
        e_steps = max(3, min(args.steps, 10))
        t0 = time.perf_counter()
        for _ in range(e_steps):
            r = e2e_step()
        ctx.synchronize()
        e_ms = (time.perf_counter() - t0) / e_steps * 1e3
        if verified is not None:
            verified = verified and w.matches(r)
        # where an end-to-end step goes: the uploads alone (every column's
        # H2D, then a wait), against the whole step
        t0 = time.perf_counter()
        for _ in range(e_steps):
            for tname, cname, ptr, arr, in_place in pinned:
                if not in_place:
                    _lib.check(lib.gpudb_upload_column(ctx.handle, tname.encode(), cname.encode(), C.c_void_p(ptr),
                                                       arr.shape[0], arr.itemsize), ctx.handle)
            ctx.synchronize()
        up_ms = (time.perf_counter() - t0) / e_steps * 1e3
        # ... and the query alone: the late columns still read in place from
        # host memory, the eager ones already resident, the result collected
        t0 = time.perf_counter()
        for _ in range(e_steps):
            ctx.run(q, collect=True)
        ctx.synchronize()
        run_ms = (time.perf_counter() - t0) / e_steps * 1e3
        if pg:
            e_ms = replicas.max_over_ranks(pg, [e_ms], "cuda")[0]
        d2h = sum(len(row) for row in r.rows) * 16 + 8
        in_place_bytes = late_bytes * ab.get("rows_reaching_aggregation", 0)
        e2e = {"value": rows_total / (e_ms / 1e3), "unit": "rows/s", "h2d_bytes_per_step": host_bytes + in_place_bytes,
               "d2h_bytes_per_step": d2h, "ms_per_step": e_ms,
               "uploaded_bytes": host_bytes, "read_in_place_bytes": in_place_bytes,
               "upload_ms": up_ms, "upload_gbs": host_bytes / (up_ms / 1e3) / 1e9, "query_ms": run_ms,
               "read_in_place_columns": sorted(f"{t}.{c}" for t, c in late)}
        # the same through the chunked streaming entry: the streamed table's
        # copies overlap the kernels of earlier chunks (and its late columns'
        # in-place reads overlap later chunks' copies)
        stune = w.stream_tune(q.tune)
        if stune is not None and args.e2e_chunk_rows > 0:
            st = w.stream_table
            qs = ctx.prepare(w.spec, stune)
            late_s = w.late_columns(stune)
            scols = [(c, ptr, arr.itemsize, (t, c) in late_s) for t, c, ptr, arr, _ in pinned if t == st]
            srows = next(arr.shape[0] for t, _, _, arr, _ in pinned if t == st)

            def stream_step():
                for tname, cname, ptr, arr, _ in pinned:
                    if tname != st:
                        _lib.check(lib.gpudb_upload_column(ctx.handle, tname.encode(), cname.encode(),
                                                           C.c_void_p(ptr), arr.shape[0], arr.itemsize), ctx.handle)
                r, _ = ctx.run_streamed(qs, st, scols, srows, args.e2e_chunk_rows)
                return r

            for _ in range(2):
                r = stream_step()
            ctx.synchronize()
            t0 = time.perf_counter()
            for _ in range(e_steps):
                r = stream_step()
            ctx.synchronize()
            s_ms = (time.perf_counter() - t0) / e_steps * 1e3
            if pg:
                s_ms = replicas.max_over_ranks(pg, [s_ms], "cuda")[0]
            s_ok = None if verified is None else w.matches(r)
            if verified is not None:
                verified = verified and s_ok
            e2e.update({"value": rows_total / (s_ms / 1e3), "ms_per_step": s_ms, "unstreamed_ms_per_step": e_ms,
                        "streamed": {"table": st, "chunk_rows": args.e2e_chunk_rows, "tune": stune,
                                     "in_place_columns": sorted(c for c, _, _, ip in scols if ip),
                                     "verified": s_ok}})
        # device copies of every column again before the host buffers go
        for tname, cname, ptr, arr, in_place in pinned:
            ctx.upload_column(tname, cname, arr)
        ctx.synchronize()
        for _, _, ptr, _, _ in pinned:
            lib.gpudb_host_free(C.c_void_p(ptr))

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        step, threads, n = time_cpu(w)
        cpu = {"value": w.rows() / step, "unit": "rows/s", "cores": threads, "kind": "port",
               "sample": f"full workload ({w.rows()} rows) x {n} runs, median"}

    line = None
    if rank == 0:
        line = {"metric": "rows_per_s", "value": value, "unit": "rows/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "int64", "data": "synthetic (seeded)",
                "config": workload_config(w, world),
                "execution": {"tune": q.tune or "default", "autotune": tuner, "cuda_graphs": not args.no_graphs,
                              "steps_enqueued_back_to_back": True},
                "verified": verified, "verified_last_timed_step": verified_timed, "phase_ms": phase_ms,
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
                "gpu_launches": launches, "clocks": clk.summary()}
    ctx.close()
    return line


def sub_args(args, **over):
    a = argparse.Namespace(**vars(args))
    for k, v in over.items():
        setattr(a, k, v)
    return a


def run_extras(args, pg, world, rank, local) -> dict:
    """The rest of the benchmark set's metric beside the headline join:
    the plain scan-filter-aggregate (config 0: q1, and the predicate
    variant q6) with their rooflines and CPU baselines, the batched mixed
    form (config 3: learned / exact / plain queries per second, checked
    against the oracle), and serving (config 4: p50 / p99 at two offered
    rates). Each part reports its own wall time and, if it fails, why."""
    import torch

    def release():
        # each part starts from the device memory the previous one held
        # handed back (its tables, arenas and pinned pools)
        gc.collect()
        torch.cuda.synchronize()
        torch.cuda.empty_cache()

    out = {}
    release()
    for which in ("q1", "q6"):
        t0 = time.perf_counter()
        try:
            # ~200 back-to-back launches of ~40 us: the host's enqueue of the
            # first one after the start event is a bubble the timed region
            # holds once, so short regions overstate the step
            a = sub_args(args, workload=which, steps=max(args.steps, 200))
            line = measure(a, make_workload(a), pg, world, rank, local)
            if line:
                out[which] = {k: line[k] for k in ("value", "unit", "ms_per_step", "config", "execution", "verified",
                                                   "verified_last_timed_step", "phase_ms", "roofline", "cpu_baseline",
                                                   "e2e", "gpu_launches", "clocks")}
                out[which]["metric"] = "rows_per_s"
                out[which]["wall_s"] = time.perf_counter() - t0
        except Exception as e:  # a failed part is reported, the headline stands
            out[which] = {"error": f"{type(e).__name__}: {e}"[:500]}
        release()
    t0 = time.perf_counter()
    try:
        line = run_mixed(sub_args(args, workload="mixed", steps=5, train_executions=args.extras_train_executions,
                                  sizer_epochs=args.extras_sizer_epochs, no_cpu_baseline=True), pg=pg)
        if line:
            line["wall_s"] = time.perf_counter() - t0
            out["mixed"] = line
    except Exception as e:
        out["mixed"] = {"error": f"{type(e).__name__}: {e}"[:500]}
    release()
    t0 = time.perf_counter()
    try:
        line = run_serve(sub_args(args, workload="serve", train_executions=args.extras_train_executions,
                                  sizer_epochs=args.extras_sizer_epochs, serve_queries=args.extras_serve_queries,
                                  serve_rates="500,2000", serve_plain_queries=100), pg=pg)
        if line:
            line["wall_s"] = time.perf_counter() - t0
            out["serve"] = line
    except Exception as e:
        out["serve"] = {"error": f"{type(e).__name__}: {e}"[:500]}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="join_topk",
                    choices=["join_topk", "q1", "q6", "q6_selvec", "groupby", "hashjoin", "mixed", "serve",
                             "aggmodes"])
    ap.add_argument("--tune", default="auto", help='tuning string, "" for the defaults, "auto" (stored or seed '
                                                   'tunings) or "search" (the full autotuner search)')
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-chunk-rows", type=int, default=8_000_000,
                    help="rows per chunk of the end-to-end streamed run (0: no streamed run)")
    ap.add_argument("--no-verify", action="store_true")
    ap.add_argument("--no-graphs", action="store_true", help="launch every kernel instead of replaying graphs")
    ap.add_argument("--no-extras", action="store_true",
                    help="the headline join only (no q1 / q6 / mixed / serve objects on the line)")
    ap.add_argument("--build-rows", type=int, default=15_000_000)
    ap.add_argument("--probe-rows", type=int, default=60_000_000)
    ap.add_argument("--fact-rows", type=int, default=6_001_215)
    ap.add_argument("--zprobe-rows", type=int, default=120_000_000)
    ap.add_argument("--zkeys", type=int, default=1 << 22)
    ap.add_argument("--mix-rows", type=int, default=120_000_000)
    ap.add_argument("--mix-dim-rows", type=int, default=1_000_000)
    ap.add_argument("--mix-queries", type=int, default=256)
    ap.add_argument("--train-executions", type=int, default=200_000)
    ap.add_argument("--sizer-epochs", type=int, default=30)
    ap.add_argument("--extras-train-executions", type=int, default=200_000)
    ap.add_argument("--extras-sizer-epochs", type=int, default=30)
    ap.add_argument("--extras-serve-queries", type=int, default=600)
    ap.add_argument("--plain-passes", type=int, default=2, help="timed passes of the plain baseline (the best is kept)")
    ap.add_argument("--agg-rows", type=int, default=0, help="aggmodes: rows of the query (default half of --zprobe-rows)")
    ap.add_argument("--agg-cards", default="", help="aggmodes: comma-separated key cardinalities")
    ap.add_argument("--agg-keys", default="", help="aggmodes: comma-separated key columns (m_rank_u, m_rank_z)")
    ap.add_argument("--batch-tune", default="", help='batch kernels\' launch shape, e.g. "block=512;tile_rows=65536"')
    ap.add_argument("--serve-rows", type=int, default=120_000_000)
    ap.add_argument("--serve-dim-rows", type=int, default=30_000_000)
    ap.add_argument("--serve-queries", type=int, default=1000)
    ap.add_argument("--serve-rates", default="500,2000,8000")
    ap.add_argument("--serve-workers", type=int, default=2)
    ap.add_argument("--serve-max-batch", type=int, default=512)
    ap.add_argument("--serve-plain-queries", type=int, default=200)
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    args.tune_search = args.tune == "search"
    if args.tune_search:
        args.tune = "auto"
    if args.workload in ("mixed", "serve", "aggmodes"):
        line = {"mixed": run_mixed, "serve": run_serve, "aggmodes": run_aggmodes}[args.workload](args)
        if line:
            print(json.dumps(line), flush=True)
        return
    world, rank, local = dist_info()
    w = make_workload(args)

    if args.impl == "reference":
        if rank == 0:
            run_reference(args, w)
        return

    import torch
    torch.cuda.set_device(local)
    from gpudbmetalcodegen_b200 import replicas
    pg = replicas.init("nccl", 120)
    line = measure(args, w, pg, world, rank, local)
    # the rest of the metric rides on the headline line of a one-GPU run
    # (under torchrun every rank would have to take the same steps)
    if args.workload == "join_topk" and not args.no_extras and world == 1:
        extras = run_extras(args, pg, world, rank, local)
        if line is not None:
            line.update(extras)
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)
    if pg:
        replicas.shutdown(pg)


if __name__ == "__main__":
    main()
