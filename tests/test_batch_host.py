"""Host-side logic of the batched / learned-sizing layer (no GPU): the C
struct layout seen from Python, the mixed-query generator, result packing,
the sizing policy, the execution log, and the MLP oracle itself (its
gradients against central finite differences)."""
import ctypes as C
import subprocess
import textwrap

import numpy as np
import pytest

from gpudbmetalcodegen_b200 import batch as B
from gpudbmetalcodegen_b200 import workloads as W
from oracle import mlp_oracle as M

from conftest import ROOT


def test_query_struct_layout_matches_header(tmp_path):
    fields = [f for f, _ in B.BatchQueryStruct._fields_]
    src = tmp_path / "layout.c"
    src.write_text(textwrap.dedent("""
        #include <stddef.h>
        #include <stdio.h>
        #include "gpudb_batch.h"
        int main(void) {
            printf("%zu\\n", sizeof(gpudb_batch_query));
        """) + "".join(f'    printf("%zu\\n", offsetof(gpudb_batch_query, {f}));\n' for f in fields) + "}\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert out[0] == C.sizeof(B.BatchQueryStruct)
    assert out[1:] == [getattr(B.BatchQueryStruct, f).offset for f in fields]


def test_mixed_query_generator():
    qs = W.gen_mixed_queries(256, seed=5)
    assert qs == W.gen_mixed_queries(256, seed=5)
    assert qs != W.gen_mixed_queries(256, seed=6)
    assert {q.tmpl for q in qs} == set(B.TEMPLATES)
    rows = np.array([q.rows for q in qs])
    assert rows.min() >= 1_000_000 and rows.max() <= 120_000_000
    # log-uniform over [1M, 120M]: median near sqrt(1M * 120M) ~ 11M
    assert 5e6 < np.median(rows) < 25e6
    for q in qs:
        assert 0 <= q.row0 and q.row0 + q.rows <= W.MIX_TABLE_ROWS
        assert 100 <= q.thr <= 9900
        assert 4 <= q.card <= 1 << 22
        assert q.key in ("m_rank_u", "m_rank_z")
        assert 0 <= q.table < len(W.MIX_ZIPF_S)
    small = W.gen_mixed_queries(50, seed=1, table_rows=10_000, min_rows=100, max_rows=5_000)
    assert all(100 <= q.rows <= 5_000 and q.row0 + q.rows <= 10_000 for q in small)


def test_unpack_results():
    qs = [B.MixQuery("agg", 0, 0, 10, 5), B.MixQuery("groupby", 0, 0, 10, 5, card=9),
          B.MixQuery("topk", 0, 0, 10, 5, card=9, k=2), B.MixQuery("join", 0, 0, 10, 5)]
    big = (1 << 70) + 12345  # a sum beyond int64: lo / hi words
    packed = np.array([[7, big & ((1 << 64) - 1), big >> 64],
                       [5, 1, 10], [2, 3, 30],
                       [2, 30, 0], [5, 10, 0],
                       [0, 0, 0]], dtype=np.uint64).astype(np.int64)
    res = B.unpack_results(qs, np.array([1, 2, 2, 1], dtype=np.uint64), packed)
    assert res[0] == ("scalar", 7, big)
    g = B.canonical(res[1])
    assert g[0] == "groups" and list(g[1]) == [2, 5] and list(g[3]) == [30, 10]
    assert res[2] == ("topk", ((2, 30), (5, 10)))
    assert res[3] == ("scalar", 0, 0)
    assert B.same_result(res[1], B.canonical_groups([5, 2], [1, 3], [10, 30]))
    assert not B.same_result(res[1], B.canonical_groups([5, 2], [1, 3], [10, 31]))


def test_sizing_policy():
    q = B.MixQuery("groupby", 0, 0, rows=1000, thr=5000, card=100_000)
    y = lambda g: np.log2(g + 1) / B.CARD_SCALE
    assert B.groups_from_prediction(q, y(300), 1.5) == pytest.approx(450, abs=2)
    assert B.groups_from_prediction(q, y(1e6), 1.5) == 1000          # clamped to the slice rows
    q2 = B.MixQuery("groupby", 0, 0, rows=10**8, thr=5000, card=64)
    assert B.groups_from_prediction(q2, y(1e6), 1.5) == 64           # clamped to card
    assert B.groups_from_prediction(q2, -1.0, 1.5) == 1


def test_labels_and_log(tmp_path):
    qs = [B.MixQuery("groupby", 0, 0, 1000, 5000, card=64), B.MixQuery("agg", 0, 0, 1000, 5000)]
    y = B.labels(qs, np.array([500, 250]), np.array([63, 0]))
    assert y[0, 0] == pytest.approx(6 / B.CARD_SCALE) and y[0, 1] == pytest.approx(0.5)
    assert y[1, 0] == 0 and y[1, 1] == pytest.approx(0.25)
    log = B.ExecutionLog()
    log.add(np.ones((2, 16)), y)
    log.add(np.zeros((3, 16)), np.zeros((3, 2)))
    assert len(log) == 5
    log.save(tmp_path / "log.npz")
    X, Y = B.ExecutionLog.load(tmp_path / "log.npz").arrays()
    assert X.shape == (5, 16) and np.array_equal(Y[:2], y)


def test_bf16_rounding():
    x = np.array([1.0, 1 + 2 ** -8, 1 + 3 * 2 ** -8, -2.5, 1 + 2 ** -7, 3.0e38], dtype=np.float32)
    r = M.bf16_round(x)
    assert list(r[:5]) == [1.0, 1.0, 1 + 2 ** -6, -2.5, 1 + 2 ** -7]  # ties to even
    assert np.isfinite(r[5])


def test_mlp_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(3)
    p = rng.normal(0, 0.3, M.NPARAMS)
    X = rng.uniform(-1, 1, (7, 16))
    Y = rng.uniform(-1, 1, (7, 2))
    _, g = M.loss_and_grads(p, X, Y, quantize=False)
    idx = rng.choice(M.NPARAMS, 60, replace=False)
    h = 1e-6
    for i in idx:
        e = np.zeros(M.NPARAMS)
        e[i] = h
        lp, _ = M.loss_and_grads(p + e, X, Y, quantize=False)
        lm, _ = M.loss_and_grads(p - e, X, Y, quantize=False)
        assert abs((lp - lm) / (2 * h) - g[i]) <= 1e-5 * max(1.0, abs(g[i])), i


def test_adam_oracle_first_step_is_signed_lr():
    w = np.zeros(5)
    g = np.array([1.0, -2.0, 0.5, -1e-3, 3.0])
    w1, m, v = M.adam_step(w, np.zeros(5), np.zeros(5), g, 1, lr=0.01)
    assert np.allclose(w1, -0.01 * np.sign(g), atol=1e-7)


def test_invariant_divisor_method():
    """The multiply-high division the batch kernels use for key % card
    (Granlund & Montgomery 1994, Fig. 4.1), restated and checked exhaustively
    at the edges and on random dividends / divisors below 2^31."""
    import random

    def div(n, d):
        l = 0
        while (1 << l) < d:
            l += 1
        m = ((1 << 32) * ((1 << l) - d)) // d + 1
        assert m < (1 << 32)
        t = (n * m) >> 32
        return (t + ((n - t) >> min(l, 1))) >> max(l - 1, 0)

    rnd = random.Random(1)
    ds = [1, 2, 3, 4, 5, 7, 100, 1023, 1024, 1025, (1 << 20) + 3, (1 << 31) - 1] + \
        [rnd.randrange(1, 1 << 31) for _ in range(200)]
    for d in ds:
        for n in [0, 1, d - 1, d, d + 1, (1 << 31) - 1] + [rnd.randrange(0, 1 << 31) for _ in range(200)]:
            assert div(n, d) == n // d, (n, d)


def test_pinned_pool_recycles_buffers_when_views_die():
    import gc
    held = {}

    def alloc(n):  # host memory stands in for pinned memory here
        b = C.create_string_buffer(n)
        held[C.addressof(b)] = b
        return C.addressof(b)

    pool = B.PinnedPool(alloc=alloc, free=lambda p: held.pop(p))
    a = pool.array(1000)
    assert a.nbytes >= 1000 and a.dtype == np.int64
    a[:] = 7
    v = a[10:20]          # a view keeps the buffer alive
    del a
    gc.collect()
    assert pool._free == []
    assert (v == 7).all()
    del v
    gc.collect()
    assert len(pool._free) == 1
    b = pool.array(500)   # reuses the freed buffer
    assert len(pool._free) == 0
    del b
    gc.collect()
    pool.close()
    assert pool._free == [] and held == {}


def test_query_dtype_matches_the_struct():
    assert B.QUERY_DTYPE.itemsize == C.sizeof(B.BatchQueryStruct)
    for name, _ in B.BatchQueryStruct._fields_:
        assert B.QUERY_DTYPE.fields[name][1] == getattr(B.BatchQueryStruct, name).offset


def test_result_fingerprint_is_order_independent_and_sensitive():
    raw = np.array([[5, 1, 10], [2, 3, 30], [9, 2, 7]], dtype=np.int64)
    a = ("groups_raw", raw)
    b = B.canonical_groups([9, 5, 2], [2, 1, 3], [7, 10, 30])
    assert B.result_fingerprint(a) == B.result_fingerprint(b)
    c = ("groups_raw", np.array([[5, 1, 10], [2, 3, 31], [9, 2, 7]], dtype=np.int64))
    assert B.result_fingerprint(a) != B.result_fingerprint(c)
    assert B.result_fingerprint(("scalar", 3, 4)) == ("scalar", 3, 4)


def test_aggregation_strategy_policy():
    f = np.zeros(16, dtype=np.float32)
    # a key domain of at most 1024 values indexes the shared table directly
    assert B.agg_mode_for(5, f, card=1) == B.AGG_SHARED_DIRECT
    assert B.agg_mode_for(1000, f, card=B.DIRECT_MAX_CARD) == B.AGG_SHARED_DIRECT
    assert B.agg_mode_for(1000, f, card=B.DIRECT_MAX_CARD + 1) == B.AGG_SHARED
    # ... unless one key holds well above its uniform share
    f[12] = 0.07  # uniform over 16 keys: 1/16 plus sampling noise
    assert B.agg_mode_for(16, f, card=16) == B.AGG_SHARED_DIRECT
    f[12] = 0.18  # Zipf(1.1) ranks modulo 16
    assert B.agg_mode_for(16, f, card=16) == B.AGG_SHARED
    f[12] = 0.003  # uniform over 1024 keys
    assert B.agg_mode_for(1024, f, card=1024) == B.AGG_SHARED_DIRECT
    f[12] = 0.0
    # beyond it: few groups or skewed keys -> shared, else the global table
    assert B.agg_mode_for(1 << 20, f, card=1 << 22) == B.AGG_GLOBAL
    f[12] = B.SKEW_SHARE
    assert B.agg_mode_for(1 << 20, f, card=1 << 22) == B.AGG_SHARED
    assert B.agg_mode_for(1 << 20, None, card=1 << 22) == B.AGG_SHARED
