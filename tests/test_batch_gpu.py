"""GPU: the batched mixed-query kernels and the learned sizer.

* every batched query (all four templates, edge cases included) equals the
  CPU oracle bit-exactly, and equals the plain one-query-at-a-time engine
  path; undersized tables are detected on the device and re-run exactly;
* the sizer's forward, gradients and Adam update equal the CPU oracle of the
  network (BF16 weights; FP32 vs float64 accumulation: tolerances below);
* the trained sizer beats the closed-form sample estimate it replaces and
  lets the batch skip the exact count pass at identical results.
"""
import numpy as np
import pytest

from gpudbmetalcodegen_b200 import batch as B
from gpudbmetalcodegen_b200 import workloads as W
from oracle import mlp_oracle as M
from oracle import oracle_py as O
from mix_oracle import oracle_result

pytestmark = pytest.mark.gpu

GRAD_RTOL = 2e-3   # |g_gpu - g_cpu| <= GRAD_RTOL * max|g_cpu| + 1e-7, per parameter tensor
FWD_RTOL = 1e-4


@pytest.fixture(scope="module")
def tables():
    return B.MixTables(rows=2_000_000, zipf_s=(0.8, 1.3), nranks=1 << 20, dim_rows=50_000, seed=77, host=True)


def edge_queries(rows):
    return [
        B.MixQuery("agg", 0, 0, 1, 10_000),                            # one row
        B.MixQuery("agg", 1, 17, 12_345, 0),                           # nothing passes
        B.MixQuery("join", 0, 3, 100_001, 9_999, attr_lt=0),           # empty build side
        B.MixQuery("join", 1, 0, rows, 10_000, attr_lt=1000),          # everything joins
        B.MixQuery("groupby", 0, 5, 77_777, 0, card=100),               # no groups
        B.MixQuery("groupby", 1, 0, rows, 10_000, key="m_rank_z", card=1),   # one group
        B.MixQuery("groupby", 0, 1, 1_000_003, 5_000, card=1 << 20),    # ~all keys distinct
        B.MixQuery("topk", 1, 9, 300_000, 7_000, key="m_rank_z", card=3, k=16),  # k > groups
        B.MixQuery("topk", 0, 0, rows, 2_500, card=1 << 16, k=1),
        B.MixQuery("topk", 1, 11, 500_000, 5_000, key="m_rank_z", card=1 << 20, k=10),  # ties at the top
        B.MixQuery("groupby", 0, 2, rows - 2, 9_000, card=1024),        # the direct table's largest domain
        B.MixQuery("groupby", 1, 0, rows, 6_000, key="m_rank_z", card=1025),  # one past it: hashed
    ]


def mixed(tables, n, seed, **kw):
    return W.gen_mixed_queries(n, seed=seed, table_rows=tables.rows, n_tables=len(tables.zipf_s),
                               min_rows=10_000, max_rows=tables.rows, max_card=1 << 20, **kw)


def assert_all_equal(got, expect, queries):
    bad = [(i, queries[i], B.describe_difference(g, e)) for i, (g, e) in enumerate(zip(got, expect))
           if not B.same_result(g, e)]
    assert not bad, bad[:3]


@pytest.mark.parametrize("use_graph", [False, True])
def test_batch_exact_sizing_matches_oracle(tables, use_graph):
    qs = edge_queries(tables.rows) + mixed(tables, 40, seed=1)
    r = B.BatchRunner(tables, sizing="exact", use_graph=use_graph)
    got, rep = r.run(qs)
    assert rep.overflowed == []
    assert_all_equal(got, [oracle_result(tables, q) for q in qs], qs)
    again, _ = r.run(qs)  # graph replay / re-execution of the same batch
    assert_all_equal(again, got, qs)
    assert rep.launches >= 3
    r.close()


@pytest.mark.parametrize("tuning", [dict(block=256, tile_rows=4096, warp_aggregate=False, max_probe=64),
                                    dict(block=1024, tile_rows=65536, warp_aggregate=True, max_probe=256),
                                    dict(block=512, tile_rows=16384, group_rows=2, agg_rows=4),
                                    dict(block=512, tile_rows=16384, group_rows=4, shared_warp=0)])
def test_batch_tunings_and_bound_sizing(tables, tuning):
    qs = mixed(tables, 32, seed=2)
    r = B.BatchRunner(tables, sizing="bound", tuning=tuning)
    got, rep = r.run(qs)
    assert rep.overflowed == []
    assert_all_equal(got, [oracle_result(tables, q) for q in qs], qs)
    r.close()


@pytest.mark.parametrize("mode", [B.AGG_SHARED, B.AGG_GLOBAL_WARP, B.AGG_GLOBAL, B.AGG_SHARED_DIRECT])
def test_every_aggregation_strategy(tables, mode):
    qs = [q for q in edge_queries(tables.rows) + mixed(tables, 80, seed=21) if q.grouped]
    r = B.BatchRunner(tables, sizing="exact", agg_mode=mode)
    got, rep = r.run(qs)
    assert rep.overflowed == []
    assert_all_equal(got, [oracle_result(tables, q) for q in qs], qs)
    r.close()


def test_exact_stats_match_numpy(tables):
    qs = edge_queries(tables.rows) + mixed(tables, 24, seed=3)
    b = B.Batch()
    b.set_queries([tables.query_struct(q) for q in qs])
    p, d, _ = b.exact_stats()
    for i, q in enumerate(qs):
        m = tables.slice_host(q)
        keep = m["m_filter"] < q.thr
        assert p[i] == keep.sum(), i
        if q.grouped:
            assert d[i] == np.unique(m[q.key][keep].astype(np.int64) % q.card).size, i
    f, _ = b.features()
    assert f.shape == (len(qs), 16) and np.isfinite(f).all()
    b.close()


def test_undersized_tables_overflow_and_rerun_exactly(ctx, tables):
    qs = [q for q in mixed(tables, 40, seed=4) if q.grouped][:12]
    plain = B.PlainRunner(ctx, tables)

    class Tiny(B.BatchRunner):
        def size(self, queries, report):  # a deliberately wrong predictor: 1 group each
            return [1] * len(queries)

    r = Tiny(tables, sizing="exact", plain=plain)
    got, rep = r.run(qs)
    expect = [oracle_result(tables, q) for q in qs]
    assert len(rep.overflowed) > 0
    # every overflowed query really has more groups than a 16-slot table holds
    for i in rep.overflowed:
        assert expect[i][0] == "topk" or expect[i][1].size > 16
    assert_all_equal(got, expect, qs)
    r.close()


def test_batch_equals_plain_path(ctx, tables):
    qs = edge_queries(tables.rows)[:8] + mixed(tables, 16, seed=5)
    plain = B.PlainRunner(ctx, tables)
    expect = [plain.run(q) for q in qs]
    r = B.BatchRunner(tables, sizing="exact")
    got, _ = r.run(qs)
    assert_all_equal(got, expect, qs)
    r.close()


def test_plain_path_buffers_keep_their_allocation(ctx, tables):
    """The plain path sizes its group table per query. A large query, a
    small one, then one in between: the later two reuse the first
    allocation (its capacity is kept apart from each run's logical size, so
    a smaller run does not make the next larger one free and allocate
    again), the logical sizes follow the queries, and every answer equals
    the oracle's."""
    import ctypes as C
    from gpudbmetalcodegen_b200 import _lib
    lib = _lib.load()
    plain = B.PlainRunner(ctx, tables)
    qs = [B.MixQuery("groupby", 0, 0, tables.rows, 10_000, card=1 << 20),
          B.MixQuery("groupby", 0, 5, 100_000, 10_000, card=1 << 20),
          B.MixQuery("groupby", 0, 7, 1_000_000, 10_000, card=1 << 20)]
    got, bufs = [], []
    for q in qs:
        got.append(plain.run(q))
        p, n = C.c_void_p(), C.c_uint64()
        assert lib.gpudb_buffer_ptr(ctx.handle, b"mg_keys", C.byref(p), C.byref(n)) == 0
        bufs.append((p.value, n.value))
    assert bufs[1][0] == bufs[0][0] and bufs[2][0] == bufs[0][0]
    assert bufs[1][1] < bufs[2][1] <= bufs[0][1]
    assert_all_equal(got, [oracle_result(tables, q) for q in qs], qs)


def test_graph_cache_captures_recurring_runs_and_ages_out(ctx, tables):
    """Graphs on, 400 plain queries whose constants are launch arguments,
    each run twice: a launch sequence's first run is eager, its second is
    captured and replayed, and past the 512 graphs a context keeps the
    oldest ones are dropped (the third pass re-runs early queries whose
    graphs aged out). Every answer equals the eager run's and, on a
    subset, the oracle's."""
    qs = mixed(tables, 400, seed=41)
    plain = B.PlainRunner(ctx, tables)
    ctx.set_use_graphs(True)
    try:
        first = [plain.run(q) for q in qs]
        second = [plain.run(q) for q in qs]
        third = [plain.run(q) for q in qs[:40]]
    finally:
        ctx.set_use_graphs(False)
    assert_all_equal(second, first, qs)
    assert_all_equal(third, first[:40], qs[:40])
    assert_all_equal(first[:40], [oracle_result(tables, q) for q in qs[:40]], qs[:40])


# ---------------------------------------------------------------------------
# the sizer network
# ---------------------------------------------------------------------------
def _tensors(v):
    return M.unpack(v)


def test_sizer_gradients_match_oracle():
    rng = np.random.default_rng(11)
    s = B.Sizer(seed=5)
    p = s.params
    for n in (1, 45, 1000):  # partial tiles, one tile, many CTAs
        X = rng.uniform(-1, 1, (n, 16)).astype(np.float32)
        Y = rng.uniform(-1, 1, (n, 2)).astype(np.float32)
        g, loss = s.grads(X, Y)
        lref, gref = M.loss_and_grads(p, X, Y)
        assert abs(loss - lref) <= 1e-4 * abs(lref) + 1e-7
        for name, a in _tensors(g).items():
            b = _tensors(gref)[name]
            assert np.abs(a - b).max() <= GRAD_RTOL * np.abs(b).max() + 1e-7, (n, name)
    s.close()


def test_sizer_forward_matches_oracle():
    rng = np.random.default_rng(12)
    s = B.Sizer(seed=6)
    p = rng.normal(0, 0.2, M.NPARAMS).astype(np.float32)
    s.params = p
    assert np.array_equal(s.params, p)
    X = rng.uniform(-1, 1, (333, 16)).astype(np.float32)
    y, _ = M.forward(p, X)
    got = s.predict(X)
    assert np.abs(got - y).max() <= FWD_RTOL * max(1.0, np.abs(y).max())
    s.close()


def test_sizer_adam_step_matches_oracle():
    rng = np.random.default_rng(13)
    s = B.Sizer(seed=7)
    p0 = s.params.astype(np.float64)
    X = rng.uniform(-1, 1, (256, 16)).astype(np.float32)
    Y = rng.uniform(-1, 1, (256, 2)).astype(np.float32)
    _, g = M.loss_and_grads(p0, X, Y)
    s.train(X, Y, epochs=1, batch=256, lr=1e-3, seed=0)  # one step over the whole set
    w1, _, _ = M.adam_step(p0, np.zeros_like(p0), np.zeros_like(p0), g, 1, lr=1e-3)
    got = s.params
    sure = np.abs(g) > 1e-5 * np.abs(g).max()  # skip gradients at the FP32 noise floor
    assert np.abs(got - w1)[sure].max() <= 2e-6
    s.close()


def test_sizer_training_reduces_loss():
    rng = np.random.default_rng(14)
    X = rng.uniform(0, 1, (4096, 16)).astype(np.float32)
    Y = np.stack([0.5 * X[:, 0] + 0.3 * X[:, 5] ** 2, np.sin(3 * X[:, 2]) * 0.2 + 0.4], 1).astype(np.float32)
    s = B.Sizer(seed=8)
    _, before = s.grads(X, Y)
    after = s.train(X, Y, epochs=40, batch=128, lr=3e-3, seed=1)
    _, final = s.grads(X, Y)
    assert final < 0.1 * before and after < 0.1 * before
    s.close()


# ---------------------------------------------------------------------------
# the gain: learned sizing vs the methods without it
# ---------------------------------------------------------------------------
def test_learned_sizer_gain(ctx, tables):
    train_q = mixed(tables, 6000, seed=100, templates=("groupby", "topk", "groupby", "topk", "agg", "join"))
    log = B.ExecutionLog()
    B.log_executions(tables, train_q, log, batch_size=1000)
    assert len(log) == 6000
    sizer, info = B.train_sizer(log, seed=3, epochs=60, batch=256, lr=2e-3)
    # the network predicts group cardinality better than the closed-form
    # estimate from the same 4096-row sample
    assert info["log2_err_net_mean"] < 0.7 * info["log2_err_estimate_mean"], info
    qs = mixed(tables, 64, seed=101)
    plain = B.PlainRunner(ctx, tables)
    runs = {}
    for sizing in ("exact", "bound", "learned"):
        r = B.BatchRunner(tables, sizing=sizing, sizer=sizer, plain=plain)
        r.run(qs)  # warm
        runs[sizing] = r.run(qs)
        r.close()
    expect = [oracle_result(tables, q) for q in qs]
    for sizing, (res, rep) in runs.items():
        assert_all_equal(res, expect, qs)
    learned, exact, bound = runs["learned"][1], runs["exact"][1], runs["bound"][1]
    # no count pass; tables within 2x of exact sizing and smaller than the
    # exact upper bound min(card, rows) that needs no pass either
    assert learned.stats_ms == 0.0 and exact.stats_ms > 0.0
    assert learned.table_slots <= 2 * exact.table_slots
    assert learned.table_slots < bound.table_slots
    assert len(learned.overflowed) <= 2
    sizer.close()


def test_device_generators_match_host():
    import torch
    from gpudbmetalcodegen_b200 import _lib
    lib = _lib.load_datagen()
    for s, row0, n in ((0.8, 0, 100_000), (1.3, 123_456_789, 77_777)):
        host = W.gen_mix(n, nranks=1 << 20, s=s, dim_rows=5000, seed=9, row0=row0)
        dev = {c: torch.empty(n, dtype={np.int32: torch.int32, np.int64: torch.int64}[dt], device="cuda")
               for c, dt in W.MIX_COLUMNS.items()}
        assert lib.gpudb_gen_mix_device(9, 1 << 20, s, 5000, row0, n, *(dev[c].data_ptr() for c in W.MIX_COLUMNS),
                                        None) == 0
        for c in W.MIX_COLUMNS:
            assert np.array_equal(dev[c].cpu().numpy(), host[c]), c
    md = W.gen_mixdim(30_000, seed=4)
    k = torch.empty(30_000, dtype=torch.int32, device="cuda")
    a = torch.empty(30_000, dtype=torch.int32, device="cuda")
    assert lib.gpudb_gen_mixdim_device(4, 0, 30_000, k.data_ptr(), a.data_ptr(), None) == 0
    assert np.array_equal(k.cpu().numpy(), md["md_key"]) and np.array_equal(a.cpu().numpy(), md["md_attr"])


def test_stage_times(tables):
    qs = mixed(tables, 16, seed=9)
    b = B.Batch()
    b.set_queries([tables.query_struct(q, groups=q.card) for q in qs])
    b.execute(use_graph=False)
    st = b.stage_ms()
    assert set(st) == set(B.Batch.STAGES) and all(v >= 0 for v in st.values())
    b.close()


def test_query_array_equals_structs(tables):
    qs = edge_queries(tables.rows) + mixed(tables, 30, seed=17)
    arr = tables.query_array(qs)
    for i, q in enumerate(qs):
        st = tables.query_struct(q)
        for name, _ in B.BatchQueryStruct._fields_:
            a, s = arr[i][name], getattr(st, name)
            assert int(a) == int(s or 0), (i, name, a, s)


def test_column_minmax_kernel_matches_numpy():
    """The zone-map kernel behind the sizer's column features (int32 and
    int64, ragged lengths, negative values, empty)."""
    import torch
    from gpudbmetalcodegen_b200.batch import column_minmax
    rng = np.random.default_rng(5)
    for n, dt in ((1, np.int32), (1025, np.int32), (300_001, np.int64), (7, np.int64)):
        a = rng.integers(-(1 << 40) if dt == np.int64 else -(1 << 30), 1 << 30, n).astype(dt)
        t = torch.from_numpy(a).cuda()
        assert column_minmax(t) == (int(a.min()), int(a.max()))
    assert column_minmax(torch.empty(0, dtype=torch.int32, device="cuda")) == (0, 0)
