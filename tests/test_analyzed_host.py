"""Analyzed queries on the CPU (no GPU): the reference's planning input built
through the C-ABI, its expressions lowered to the engine's exact fixed
point, every supported shape planned and compiled for sm_100a, and every
unsupported one refused with a reason."""
import pytest

from gpudbmetalcodegen_b200 import analyzed as A
from gpudbmetalcodegen_b200._lib import GpudbError


def li(aq, c):
    return aq.col("lineitem", c)


def q1_query():
    """The reference harness's Q1 analysis (lineitem names, float literals)."""
    aq = A.AnalyzedQuery()
    aq.table("lineitem")
    aq.filter(aq.cmp(A.LE, li(aq, "l_shipdate"), aq.lit(2436)))
    aq.group_by(li(aq, "l_returnflag")).group_by(li(aq, "l_linestatus"))
    one = aq.litf(1.0)
    price, disc = li(aq, "l_extendedprice"), li(aq, "l_discount")
    dp = aq.binary(A.MUL, price, aq.binary(A.SUB, one, disc))
    aq.agg(A.SUM, li(aq, "l_quantity"), "sum_qty").agg(A.SUM, price, "sum_base_price")
    aq.agg(A.SUM, dp, "sum_disc_price")
    aq.agg(A.SUM, aq.binary(A.MUL, dp, aq.binary(A.ADD, one, li(aq, "l_tax"))), "sum_charge")
    return aq


def q6_query(qty_lt=24, disc=(0.05, 0.07), ship=(365, 730)):
    aq = A.AnalyzedQuery()
    aq.table("lineitem")
    s = li(aq, "l_shipdate")
    aq.filter(aq.cmp(A.GE, s, aq.lit(ship[0]))).filter(aq.cmp(A.LT, s, aq.lit(ship[1])))
    aq.filter(aq.between(li(aq, "l_discount"), aq.litf(disc[0]), aq.litf(disc[1])))
    aq.filter(aq.cmp(A.LT, li(aq, "l_quantity"), aq.lit(qty_lt)))
    aq.agg(A.SUM, aq.binary(A.MUL, li(aq, "l_extendedprice"), li(aq, "l_discount")), "revenue")
    return aq


def test_lowering_tracks_decimal_scales_exactly():
    aq = q1_query()
    one = aq.litf(1.0)
    price, disc, tax = li(aq, "l_extendedprice"), li(aq, "l_discount"), li(aq, "l_tax")
    dp = aq.binary(A.MUL, price, aq.binary(A.SUB, one, disc))
    assert aq.lower(dp) == ("(f_price[i] * (100ll - f_discount[i]))", 4)
    assert aq.lower(aq.binary(A.MUL, dp, aq.binary(A.ADD, one, tax)))[1] == 6
    # single-precision noise in a decimal literal still lowers exactly
    assert aq.lower_pred(aq.between(disc, aq.litf(0.05000000074505806), aq.litf(0.07))) == \
        "(f_discount[i] >= 5ll && f_discount[i] <= 7ll)"
    # a literal finer than the column scales the column up, not the literal down
    assert aq.lower_pred(aq.cmp(A.LT, disc, aq.litf(0.055))) == "(f_discount[i] * 10ll) < 55ll"
    assert aq.lower_pred(aq.cmp(A.EQ, li(aq, "l_returnflag"), aq.lits("R"))) == "f_flag_a[i] == 'R'"
    assert aq.lower_pred(aq.in_list(li(aq, "l_quantity"), [aq.lit(1), aq.lit(3)])) == \
        "(f_quantity[i] == 1ll || f_quantity[i] == 3ll)"
    assert aq.lower_pred(aq.not_(aq.or_(aq.cmp(A.GT, li(aq, "l_tax"), aq.litf(0.04)),
                                        aq.cmp(A.EQ, li(aq, "l_quantity"), aq.lit(7))))) == \
        "!(((f_tax[i] > 4ll) || (f_quantity[i] == 7ll)))"
    # engine names resolve directly, and integer arithmetic keeps scale 0
    assert aq.lower(aq.binary(A.ADD, aq.col("fact", "f_quantity"), aq.lit(3))) == ("(f_quantity[i] + 3ll)", 0)


@pytest.mark.parametrize("build", [
    lambda aq: aq.lower(aq.binary(A.DIV, li(aq, "l_extendedprice"), aq.lit(2))),          # division
    lambda aq: aq.lower(aq.col("lineitem", "l_comment")),                                  # unknown column
    lambda aq: aq.lower(aq.binary(A.ADD, li(aq, "l_returnflag"), aq.lit(1))),              # char arithmetic
    lambda aq: aq.lower_pred(aq.cmp(A.EQ, li(aq, "l_returnflag"), aq.lit(65))),            # char vs number
    lambda aq: aq.lower_pred(aq.cmp(A.LT, li(aq, "l_discount"), aq.litf(1e-20))),          # not exact
    lambda aq: aq.lower(aq.lits("AB")),                                                    # multi-char
])
def test_what_has_no_exact_lowering_is_refused(build):
    with pytest.raises(GpudbError):
        build(A.AnalyzedQuery())


def test_foreign_or_null_nodes_are_rejected():
    a, b = A.AnalyzedQuery(), A.AnalyzedQuery()
    x = a.col("fact", "f_quantity")
    with pytest.raises(GpudbError):
        b.binary(A.ADD, x, b.lit(1))
    with pytest.raises(GpudbError):
        b.filter(a.cmp(A.LT, x, a.lit(3)))
    with pytest.raises(GpudbError):
        a.agg(A.SUM, None, "s")  # only COUNT(*) has no expression


def test_shapes_plan_and_compile():
    q = q1_query().prepare(None, "Q1")
    assert "KeyedAgg(d_ir_keyed, 6 buckets, 4 aggs" in q.plan
    q = q6_query().prepare(None, "Q6")
    assert "TGReduce(1 accumulators)" in q.plan and "f_discount[i] >= 5ll" in q.source
    # Q18 shape: one integer GROUP BY column -> hash group-by
    aq = A.AnalyzedQuery().table("zprobe")
    k = aq.col("zprobe", "z_key")
    aq.group_by(k).target(k).agg(A.SUM, aq.col("zprobe", "z_value"), "sum").agg(A.COUNT, None, "count")
    assert "HashGroupBy(irg, key=(long long)z_key[i]" in aq.prepare(None, "Q18").plan
    # Q3 shape: dim JOIN probe, GROUP BY the key, ORDER BY the sum DESC LIMIT k
    assert "JT_topk" in join_query(k=10).prepare(None, "Q3").plan
    assert "JT_probe_group" in join_query(k=-1).prepare(None, "Q3all").plan


def join_query(k=10, seg=1, od_lt=1170, ship_gt=1170):
    aq = A.AnalyzedQuery().table("dim").table("probe").join("dim", "b_key", "probe", "p_fk")
    aq.filter(aq.cmp(A.EQ, aq.col("dim", "b_segment"), aq.lit(seg)))
    aq.filter(aq.cmp(A.LT, aq.col("dim", "b_order_day"), aq.lit(od_lt)))
    aq.filter(aq.cmp(A.GT, aq.col("probe", "p_ship_day"), aq.lit(ship_gt)))
    key = aq.col("probe", "p_fk")
    rev = aq.binary(A.MUL, aq.col("probe", "p_price"), aq.binary(A.SUB, aq.litf(1.0), aq.col("probe", "p_discount")))
    aq.group_by(key).target(key).agg(A.SUM, rev, "revenue")
    if k > 0:
        aq.order_by(aq.ref("revenue"), True).order_by(aq.col("probe", "p_fk")).limit(k)
    return aq


@pytest.mark.parametrize("mutate,msg", [
    (lambda aq: aq.table("mix"), "more than two tables"),
    (lambda aq: aq.limit(5), "ORDER BY"),
    (lambda aq: aq.agg(A.MIN, aq.col("lineitem", "l_quantity"), "m"), "MIN"),
])
def test_unplannable_shapes_name_the_reason(mutate, msg):
    aq = q6_query()
    if msg == "more than two tables":
        aq.table("dim").table("probe")
    mutate(aq)
    with pytest.raises(GpudbError) as e:
        aq.prepare(None, "X")
    assert msg in e.value.message
    with pytest.raises(GpudbError) as e:
        join_query(k=40).prepare(None, "X")
    assert "LIMIT" in e.value.message
    with pytest.raises(GpudbError) as e:
        q6_query().prepare(None, "bad name")
    assert "kernel name" in e.value.message
