"""GPU parity of the reference's other operator chains, each through the
C-ABI against the CPU oracle on the same seeded tables (bit-exact):

* join_direct — Q3's direct-address join (ArrayStore x2 -> ArrayLookup ->
  AtomicAgg), top-k over the dense array and the top keys' attributes;
* anti_join  — Q22's anti-join (BitmapBuild -> AntiBitmapProbe ->
  ComputeExpr -> AtomicCount + AtomicAgg);
* histogram  — Q13's count-of-counts (AtomicCount -> ArrayLookup ->
  AtomicCount);
* q6_selvec  — the predicate variant over a warp-built selection bitmap
  consumed by a second phase (Selection bitmap -> SelectionScan);
* multi_join — Q5's five-phase plan over a snowflake (nation bitmap ->
  customer / supplier nation maps -> orders map -> lines' double lookup,
  same-nation selection and per-nation sum);
* groupby_sorted — every group of the skewed-key group-by in ORDER BY sum
  DESC, key ASC, merge-sorted on the GPU (the reference sorts on the host).

Each runs at small sizes under several tunings, twice through the same
buffers, on edge cases (nothing qualifies, everything qualifies, ragged
row counts), and once at full size: the join configuration's tables (15M
build + 60M probe rows), the fact table (6,001,215 rows), or a snowflake of
1.5M customers, 100k suppliers, 15M orders and 60M lines.
"""
import numpy as np
import pytest

from gpudbmetalcodegen_b200 import workloads as W
from gpudbmetalcodegen_b200._lib import GpudbError
from oracle import oracle_py as O

pytestmark = pytest.mark.gpu

TUNES = ["", "scan=direct", "bs=256;stages=2;occ=3", "vec=4", "bs=1024;tile=2048;stages=3"]


def load_join(ctx, nd, npr, seed=3):
    d = W.gen_dim(nd, seed=seed)
    p = W.gen_probe(npr, dim_rows=nd, seed=seed)
    ctx.upload_table("dim", d)
    ctx.upload_table("probe", p)
    return d, p


@pytest.mark.parametrize("tune", TUNES)
def test_join_direct_parity(ctx, tune):
    d, p = load_join(ctx, 150_000, 600_000, seed=21)
    for spec, kw in (("template=join_direct", {}), ("template=join_direct;k=32;seg=3;ship_gt=900", dict(k=32, seg=3, ship_gt=900))):
        exp = O.join_direct(d, p, **kw)
        for _ in range(2):
            res, t = ctx.run(spec, tune)
            assert t.device_error == 0
            assert res.columns == ["key", "revenue", "order_day", "segment"]
            assert res.rows == exp
    # nothing qualifies on the build side: no rows
    res, _ = ctx.run("template=join_direct;od_lt=0", tune)
    assert res.rows == []


def test_join_direct_matches_join_topk_at_full_size(ctx):
    d, p = load_join(ctx, W.DIM_ROWS, W.PROBE_ROWS)
    exp = O.join_direct(d, p)
    res, t = ctx.run("template=join_direct")
    assert t.device_error == 0 and res.rows == exp
    top, _ = ctx.run("template=join_topk")
    assert [r[:2] for r in res.rows] == top.rows


@pytest.mark.parametrize("tune", TUNES)
def test_anti_join_parity(ctx, tune):
    d, p = load_join(ctx, 120_000, 500_000, seed=22)
    for spec, kw in (("template=anti_join", {}), ("template=anti_join;seg=0;od_lt=2000;ship_gt=300",
                                                  dict(seg=0, od_lt=2000, ship_gt=300)),
                     ("template=anti_join;od_lt=0", dict(od_lt=0)),  # no qualifying key: every shipped row passes
                     ("template=anti_join;ship_gt=100000", dict(ship_gt=100000))):  # no probe row ships
        exp = O.anti_join(d, p, **kw)
        for _ in range(2):
            res, t = ctx.run(spec, tune)
            assert t.device_error == 0
            assert res.columns == ["discount", "count", "sum_price"]
            assert res.rows == exp


def test_anti_join_bin_out_of_range_is_a_bounds_error(ctx):
    d = W.gen_dim(10_000, seed=5)
    p = W.gen_probe(40_000, dim_rows=10_000, seed=5)
    p["p_discount"][123] = 11  # the bin of a discount outside 0..10
    ctx.upload_table("dim", d)
    ctx.upload_table("probe", p)
    with pytest.raises(ValueError):
        O.anti_join(d, p, od_lt=0, ship_gt=-1)
    with pytest.raises(GpudbError) as e:
        ctx.run("template=anti_join;od_lt=0;ship_gt=-1")
    assert e.value.status == -7 and e.value.timing.device_error & 0x4


@pytest.mark.parametrize("tune", TUNES)
def test_histogram_parity(ctx, tune):
    d, p = load_join(ctx, 100_000, 700_000, seed=23)
    for spec, kw in (("template=histogram", {}), ("template=histogram;ship_gt=0;bins=64", dict(ship_gt=0, nbins=64)),
                     ("template=histogram;ship_gt=100000", dict(ship_gt=100000))):  # every key has 0 rows
        exp = O.histogram(d, p, **kw)
        for _ in range(2):
            res, t = ctx.run(spec, tune)
            assert t.device_error == 0
            assert res.columns == ["rows_per_key", "keys"]
            assert res.rows == exp
    # a count beyond the bins is a bounds error, as in the oracle
    with pytest.raises(ValueError):
        O.histogram(d, p, ship_gt=0, nbins=4)
    with pytest.raises(GpudbError) as e:
        ctx.run("template=histogram;ship_gt=0;bins=4", tune)
    assert e.value.timing.device_error & 0x4


def test_anti_join_and_histogram_at_full_size(ctx):
    d, p = load_join(ctx, W.DIM_ROWS, W.PROBE_ROWS)
    res, t = ctx.run("template=anti_join")
    assert t.device_error == 0 and res.rows == O.anti_join(d, p)
    res, t = ctx.run("template=histogram")
    assert t.device_error == 0 and res.rows == O.histogram(d, p)


Q6_SPECS = [("template=q6_selvec", {}), ("template=q6_selvec;ship_ge=0;ship_lt=3000;disc_lo=0;disc_hi=10;qty_lt=51",
                                          dict(ship_ge=0, ship_lt=3000, disc_lo=0, disc_hi=10, qty_lt=51)),
            ("template=q6_selvec;ship_ge=5000", dict(ship_ge=5000))]


@pytest.mark.parametrize("tune", TUNES + ["vec=2;bs=256", "pf=0;tile=1024;stages=2"])
def test_q6_selection_bitmap_parity(ctx, tune):
    f = W.gen_fact(300_000, seed=24)
    ctx.upload_table("fact", f)
    for spec, kw in Q6_SPECS:
        exp = O.q6(f, **kw)
        for _ in range(2):  # the bitmap is refilled with zeros between runs
            res, t = ctx.run(spec, tune)
            assert t.device_error == 0
            assert res.rows == [(exp,)]


@pytest.mark.parametrize("n", [1, 31, 33, 1023, 1025, 70_001])
def test_q6_selection_bitmap_ragged_rows(ctx, n):
    f = W.gen_fact(n, seed=25)
    ctx.upload_table("fact", f)
    kw = dict(ship_ge=0, ship_lt=3000, disc_lo=0, disc_hi=10, qty_lt=51)  # every row selected
    res, _ = ctx.run("template=q6_selvec;ship_ge=0;ship_lt=3000;disc_lo=0;disc_hi=10;qty_lt=51")
    assert res.rows == [(O.q6(f, **kw),)]
    # the bitmap holds exactly the selected rows
    bits = ctx.read_buffer("q6_sel", np.uint32, n // 32 + 1)
    sel = np.unpackbits(bits.view(np.uint8), bitorder="little")[:n]
    assert sel.all() and not np.unpackbits(bits.view(np.uint8), bitorder="little")[n:].any()
    res, _ = ctx.run("template=q6_selvec")
    assert res.rows == [(O.q6(f),)]


def test_q6_selection_bitmap_full_size(ctx):
    f = W.gen_fact(W.FACT_ROWS)
    ctx.upload_table("fact", f)
    res, t = ctx.run("template=q6_selvec")
    assert t.device_error == 0 and res.rows == [(O.q6(f),)]
    d = f["f_discount"]
    sel = (f["f_ship_day"] >= 365) & (f["f_ship_day"] < 730) & (d >= 5) & (d <= 7) & (f["f_quantity"] < 24)
    bits = ctx.read_buffer("q6_sel", np.uint32, W.FACT_ROWS // 32 + 1)
    assert np.array_equal(np.unpackbits(bits.view(np.uint8), bitorder="little")[:W.FACT_ROWS].astype(bool), sel)


def load_snow(ctx, scale=1.0, seed=3):
    snow = W.gen_snowflake(int(W.SNOW_CUST_ROWS * scale), int(W.SNOW_SUPP_ROWS * scale),
                           int(W.SNOW_ORDER_ROWS * scale), int(W.SNOW_LINE_ROWS * scale), seed=seed)
    for t, cols in snow.items():
        ctx.upload_table(t, cols)
    return snow


@pytest.mark.parametrize("tune", TUNES)
def test_multi_join_parity(ctx, tune):
    """The reference's Q5 plan shape: five phases (nation bitmap, two
    nation maps, the orders' map, the lines' double lookup + same-nation
    selection + per-nation sum), against the oracle for several regions and
    date ranges, twice through the same buffers."""
    snow = load_snow(ctx, scale=0.02, seed=41)
    for spec, kw in (("template=multi_join", {}), ("template=multi_join;region=0;day_ge=0;day_lt=2406",
                                                   dict(region=0, day_ge=0, day_lt=2406)),
                     ("template=multi_join;region=4;day_ge=1000;day_lt=1001", dict(region=4, day_ge=1000, day_lt=1001)),
                     ("template=multi_join;region=7", dict(region=7))):  # no nation in the region: no rows
        exp = O.multi_join(snow, **kw)
        for _ in range(2):
            res, t = ctx.run(spec, tune)
            assert t.device_error == 0
            assert res.columns == ["nation", "revenue"]
            assert res.rows == exp


def test_multi_join_full_size(ctx):
    snow = load_snow(ctx, scale=1.0, seed=W.SEED)
    res, t = ctx.run("template=multi_join")
    assert t.device_error == 0 and res.rows == O.multi_join(snow)


def sorted_groups(zp, nkeys):
    k, c, s = O.groupby(zp["z_key"], zp["z_value"], cap=nkeys)
    order = np.lexsort((k, -s))  # sum descending, then key ascending
    return [(int(k[i]), int(c[i]), int(s[i])) for i in order]


@pytest.mark.parametrize("nkeys,rows,tune", [(1 << 10, 200_000, ""), (1 << 16, 1_000_000, ""),
                                             (1 << 16, 1_000_000, "smem=0;warp=0"), (3000, 3000, ""),
                                             (1 << 14, 2_048 * 4, "bs=256"), (5, 100, "")])
def test_groupby_sorted_parity(ctx, nkeys, rows, tune):
    """ORDER BY sum DESC, key ASC over every group, sorted on the GPU
    (chunk sort + merge passes), against the oracle's groups sorted on the
    host — ragged group counts (a partial last chunk, fewer groups than one
    chunk, exactly whole chunks) and several merge depths."""
    zp = W.gen_zprobe(rows, nkeys=nkeys, s=1.1, seed=51)
    ctx.upload_table("zprobe", zp)
    ctx.register_symbol("zgroups", nkeys)
    for _ in range(2):
        res, t = ctx.run("template=groupby_sorted", tune)
        assert t.device_error == 0
        assert res.columns == ["key", "count", "sum"]
        assert res.rows == sorted_groups(zp, nkeys)


def test_groupby_sorted_full_size(ctx):
    """120M Zipf(1.1) rows over 2^22 keys: ~3.3M groups, eleven merge passes."""
    nkeys = 1 << 22
    zp = W.gen_zprobe(120_000_000, nkeys=nkeys, s=1.1, seed=W.SEED)
    ctx.upload_table("zprobe", zp)
    ctx.register_symbol("zgroups", nkeys)
    res, t = ctx.run("template=groupby_sorted", "", arrays=True)
    assert t.device_error == 0
    k, c, s = O.groupby(zp["z_key"], zp["z_value"], cap=nkeys)
    order = np.lexsort((k, -s))
    assert np.array_equal(res["key"], k[order])
    assert np.array_equal(res["count"], c[order])
    assert np.array_equal(res["sum"], s[order])
