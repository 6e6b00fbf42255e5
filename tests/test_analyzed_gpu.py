"""GPU: analyzed queries (the reference's planning input, built through the
C-ABI) planned, run and checked against the CPU oracle bit-exactly — the
same Q1 and Q6 analyses the reference harness hands to the reference's own
buildMetalPlan (lineitem names, float literals), the Q3-shape join with a
GPU top-k and with every group, the Q18-shape hash group-by, and AVG /
COUNT in a keyed aggregate."""
import numpy as np
import pytest

from gpudbmetalcodegen_b200 import analyzed as A
from gpudbmetalcodegen_b200 import workloads as W
from oracle import oracle_py as O
from test_analyzed_host import join_query, q1_query, q6_query

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fact():
    return W.gen_fact(400_000, seed=31)


@pytest.mark.parametrize("tune", ["", "keyed=5;bs=256;tile=512;stages=2;occ=2;vec=2", "scan=direct"])
def test_reference_q1_analysis(ctx, fact, tune):
    ctx.upload_table("fact", fact)
    q = q1_query().prepare(ctx, "Q1", tune)
    res, t = ctx.run(q)
    assert t.device_error == 0
    assert res.columns[:2] == ["l_returnflag", "l_linestatus"]
    expect = O.q1(fact)
    got = res.as_dicts()
    assert [(g["l_returnflag"], g["l_linestatus"]) for g in got] == [(e["flag_a"], e["flag_b"]) for e in expect]
    for g, e in zip(got, expect):
        for k in ("sum_qty", "sum_base_price", "sum_disc_price", "sum_charge"):
            assert g[k] == e[k], k


def test_reference_q6_analysis(ctx, fact):
    ctx.upload_table("fact", fact)
    res, _ = ctx.run(q6_query().prepare(ctx, "Q6"))
    assert res.rows == [(O.q6(fact),)]
    res, _ = ctx.run(q6_query(qty_lt=51, disc=(0.0, 0.1), ship=(0, 3000)).prepare(ctx, "Q6all"))
    assert res.rows == [(O.q6(fact, 0, 3000, 0, 10, 51),)]


def test_keyed_avg_and_count(ctx, fact):
    ctx.upload_table("fact", fact)
    aq = A.AnalyzedQuery().table("fact")
    flag = aq.col("fact", "f_flag_a")
    aq.filter(aq.cmp(A.GT, aq.col("fact", "f_tax"), aq.litf(0.02)))
    aq.group_by(flag).target(flag)
    aq.agg(A.AVG, aq.col("fact", "f_quantity"), "avg_qty").agg(A.COUNT, None, "n")
    res, _ = ctx.run(aq.prepare(ctx, "AVGQ"))
    keep = fact["f_tax"] > 2
    rows = {}
    for g in res.as_dicts():
        rows[g["f_flag_a"]] = g
    for ch in "ANR":
        sel = keep & (fact["f_flag_a"] == ord(ch))
        if not sel.any():
            assert ch not in rows
            continue
        n = int(sel.sum())
        s = int(fact["f_quantity"][sel].sum())
        assert rows[ch]["n"] == n and rows[ch]["_sum_avg_qty"] == s
        assert rows[ch]["avg_qty"] == float(s) / float(n)


def test_join_analysis_top_k_and_all_groups(ctx):
    d = W.gen_dim(100_000, seed=33)
    p = W.gen_probe(400_000, dim_rows=100_000, seed=33)
    ctx.upload_table("dim", d)
    ctx.upload_table("probe", p)
    res, _ = ctx.run(join_query(k=10).prepare(ctx, "Q3"))
    assert res.rows == O.join_topk(d, p, k=10)[0]
    res, _ = ctx.run(join_query(k=7, seg=2, od_lt=900, ship_gt=1000).prepare(ctx, "Q3b"))
    assert res.rows == O.join_topk(d, p, seg=2, od_lt=900, ship_gt=1000, k=7)[0]
    res, _ = ctx.run(join_query(k=-1).prepare(ctx, "Q3all"))
    sums = {}
    for _, k, v in O.join_rows(d, p):
        sums[k] = sums.get(k, 0) + v
    assert res.rows == sorted(sums.items())


def test_hash_groupby_analysis(ctx):
    nkeys = 1 << 14
    zp = W.gen_zprobe(300_000, nkeys=nkeys, s=1.1, seed=34)
    ctx.upload_table("zprobe", zp)
    aq = A.AnalyzedQuery().table("zprobe")
    k = aq.col("zprobe", "z_key")
    aq.group_by(k).target(k).agg(A.COUNT, None, "count").agg(A.SUM, aq.col("zprobe", "z_value"), "sum")
    res, t = ctx.run(aq.prepare(ctx, "Q18"))
    assert t.device_error == 0
    ek, ec, es = O.groupby(zp["z_key"], zp["z_value"], cap=nkeys)
    assert np.array_equal(np.array(res.column("z_key")), ek)
    assert np.array_equal(np.array(res.column("count")), ec)
    assert np.array_equal(np.array(res.column("sum")), es)
