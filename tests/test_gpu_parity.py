"""GPU parity: every generated pipeline, called through the C-ABI, against
the CPU oracle on the same seeded inputs. Integers must match bit-exactly;
FP64 derived averages to 1e-12 relative (they are the same IEEE division of
the same exact integers, so they are in fact identical)."""
import numpy as np
import pytest

from gpudbmetalcodegen_b200 import workloads as W
from gpudbmetalcodegen_b200._lib import GpudbError, DEVERR_HASH_OVERFLOW
from oracle import oracle_py as O

pytestmark = pytest.mark.gpu
REL = 1e-12

Q1_TUNES = ["", "scan=direct", "bs=256;tile=1024;stages=2", "bs=1024;tile=2048;stages=3", "bs=128;tile=512;stages=8",
            "keyed=1", "keyed=2", "keyed=3", "keyed=4;occ=2", "bs=256;occ=3", "vec=4", "vec=2;bs=256", "vec=8;tile=2048",
            "keyed=5;bs=256;tile=512;stages=2;occ=2", "keyed=5;scan=direct", "keyed=5;bs=128;tile=256;occ=3",
            "keyed=5;vec=2;bs=256;tile=512;stages=2", "keyed=5;vec=4;bs=256;tile=512;stages=2", "keyed=5;bs=512;tile=512;stages=2"]


def assert_q1_equal(res, expect):
    got = res.as_dicts()
    assert [(r["flag_a"], r["flag_b"]) for r in got] == [(r["flag_a"], r["flag_b"]) for r in expect]
    for g, e in zip(got, expect):
        for k in O.Q1_AGGS:
            assert g[k] == e[k], (k, g[k], e[k])
        for k in ("avg_qty", "avg_price", "avg_disc"):
            assert abs(g[k] - e[k]) <= REL * abs(e[k]), (k, g[k], e[k])


@pytest.fixture(scope="module")
def fact_small():
    return W.gen_fact(300_000, seed=11)


@pytest.mark.parametrize("tune", Q1_TUNES)
def test_q1_parity(ctx, fact_small, tune):
    ctx.upload_table("fact", fact_small)
    res, t = ctx.run("template=q1", tune)
    assert t.device_error == 0
    assert_q1_equal(res, O.q1(fact_small))


@pytest.mark.parametrize("tune", ["", "scan=direct", "bs=1024;tile=4096;stages=2", "vec=4", "vec=8;bs=256"])
def test_q6_parity(ctx, fact_small, tune):
    ctx.upload_table("fact", fact_small)
    res, _ = ctx.run("template=q6", tune)
    assert res.rows == [(O.q6(fact_small),)]
    res, _ = ctx.run("template=q6;ship_ge=0;ship_lt=3000;disc_lo=0;disc_hi=10;qty_lt=51", tune)
    assert res.rows == [(O.q6(fact_small, 0, 3000, 0, 10, 51),)]


@pytest.mark.parametrize("n", [0, 1, 15, 1023, 1025, 4097, 70_001])
def test_q1_ragged_and_empty_tables(ctx, n):
    f = W.gen_fact(n, seed=5)
    ctx.upload_table("fact", f)
    res, _ = ctx.run("template=q1")
    expect = O.q1(f)
    if n == 0:
        assert res.rows == [] and expect == []
    else:
        assert_q1_equal(res, expect)


def test_q1_filter_rejects_everything(ctx, fact_small):
    ctx.upload_table("fact", fact_small)
    res, _ = ctx.run("template=q1;ship_le=-1")
    assert res.rows == []


def test_q1_misaligned_columns_fall_back_to_direct_loads(ctx):
    torch = pytest.importorskip("torch")
    f = W.gen_fact(50_001, seed=9)
    keep = {}
    for name, arr in f.items():
        t = torch.from_numpy(arr).cuda()
        keep[name] = t
        # rows 1..n: the u8 columns start 1 byte past a 16-byte boundary
        ctx.register_column("fact", name, t.data_ptr() + arr.itemsize, arr.shape[0] - 1, arr.itemsize)
    torch.cuda.synchronize()
    sub = {k: v[1:] for k, v in f.items()}
    for tune in ("", "keyed=5", "keyed=4"):
        res, _ = ctx.run("template=q1", tune)
        assert_q1_equal(res, O.q1(sub))
    del keep


def test_q1_full_size(ctx):
    f = W.gen_fact(W.FACT_ROWS)
    ctx.upload_table("fact", f)
    for tune in ("", "scan=direct", "keyed=5;bs=256;tile=512;stages=2;occ=2", "keyed=4;bs=256;stages=2;occ=2"):
        res, _ = ctx.run("template=q1", tune)
        assert_q1_equal(res, O.q1(f))
    res, _ = ctx.run("template=q6")
    assert res.rows == [(O.q6(f),)]


# ---------------------------------------------------------------------------
# join + group + top-k
# ---------------------------------------------------------------------------
def load_join(ctx, nd, npr, seed=3):
    d = W.gen_dim(nd, seed=seed)
    p = W.gen_probe(npr, dim_rows=nd, seed=seed)
    ctx.upload_table("dim", d)
    ctx.upload_table("probe", p)
    return d, p


@pytest.mark.parametrize("tune", ["", "scan=direct", "bs=256", "split=0", "split=0;warp=0", "split=0;late=0",
                                  "split=0;bs=1024;tile=2048;stages=3", "split=0;vec=4;pf=4", "split=0;vec=8;late=0",
                                  "vec=4", "pf=4", "stages=2;warp=0;occ=4", "bvec=4;bbs=256"])
def test_join_topk_parity(ctx, tune):
    d, p = load_join(ctx, 200_000, 800_000)
    top, groups, distinct = O.join_topk(d, p, k=10)
    res, t = ctx.run("template=join_topk", tune)
    assert t.device_error == 0
    assert res.rows == top
    if "split=0" not in tune:
        # sized on the device from min(matched rows, qualifying build keys):
        # no host sizing symbol; the table holds exactly the joined groups
        assert int(ctx.read_buffer("jg_nslots", np.uint64, 1)[0]) == groups
        assert int(ctx.read_buffer("jb_distinct", np.uint64, 1)[0]) == distinct
    else:
        assert ctx.get_symbol("jt_groups") == distinct
    res, _ = ctx.run("template=join_topk;k=32")
    assert res.rows == O.join_topk(d, p, k=32)[0]


@pytest.mark.parametrize("ship_gt,od_lt", [(10**6, 1170), (1170, 0), (2555, 1170), (1170, 1170)])
def test_split_join_device_sizing_edges(ctx, ship_gt, od_lt):
    """The split plan sizes its group table on the device: no matched rows,
    no qualifying build keys, very few matches, and the default case, each
    against the oracle, run twice through the same buffers (a smaller
    second query must not see the first one's groups)."""
    d, p = load_join(ctx, 50_000, 300_000, seed=9)
    spec = f"template=join_topk;ship_gt={ship_gt};od_lt={od_lt}"
    for tune in ("split=1", "split=1;stages=2;occ=3"):
        top, groups, _ = O.join_topk(d, p, ship_gt=ship_gt, od_lt=od_lt, k=10)
        big, _ = ctx.run("template=join_topk;ship_gt=0", tune)
        assert big.rows == O.join_topk(d, p, ship_gt=0, k=10)[0]
        res, t = ctx.run(spec, tune)
        assert t.device_error == 0
        assert res.rows == top
        assert int(ctx.read_buffer("jg_nslots", np.uint64, 1)[0]) == groups


@pytest.mark.parametrize("spec,tune", [("template=join_rows", ""), ("template=join_rows;ship_gt=2000", "scan=direct"),
                                       ("template=join_rows;od_lt=0", ""), ("template=join_rows;seg=3;ship_gt=600", "bs=256")])
def test_join_rows_parity(ctx, spec, tune):
    """Materialised join output (row, key, revenue): the same multiset of
    rows as the oracle, in any order; none when nothing matches."""
    d, p = load_join(ctx, 100_000, 400_000, seed=13)
    kv = dict(x.split("=") for x in spec.split(";")[1:])
    exp = O.join_rows(d, p, seg=int(kv.get("seg", 1)), od_lt=int(kv.get("od_lt", 1170)),
                      ship_gt=int(kv.get("ship_gt", 1170)))
    for _ in range(2):  # twice through the same buffers
        res, t = ctx.run(spec, tune)
        assert t.device_error == 0
        assert sorted(res.rows) == exp
    assert res.columns == ["row", "key", "revenue"]


def test_sql_runs_through_the_templates(ctx, fact_small):
    """SELECTs over the engine's tables run through the template their
    shape maps to and give the oracle's answers."""
    d, p = load_join(ctx, 100_000, 400_000, seed=19)
    res, _ = ctx.run_sql("SELECT p_fk, SUM(p_price * (100 - p_discount)) AS revenue FROM dim, probe "
                         "WHERE b_key = p_fk AND b_segment = 2 AND b_order_day < 900 AND p_ship_day > 1000 "
                         "GROUP BY p_fk ORDER BY revenue DESC, p_fk LIMIT 7")
    assert res.rows == O.join_topk(d, p, seg=2, od_lt=900, ship_gt=1000, k=7)[0]
    ctx.upload_table("fact", fact_small)
    res, _ = ctx.run_sql("select sum(f_price * f_discount) from fact where f_ship_day >= 0 and f_ship_day < 3000 "
                         "and f_discount between 0 and 10 and f_quantity < 51")
    assert res.rows == [(O.q6(fact_small, 0, 3000, 0, 10, 51),)]


def test_join_topk_ties_break_by_key(ctx):
    # every probe row carries the same revenue: ranking is decided by key
    d = W.gen_dim(5000, seed=4)
    p = W.gen_probe(20_000, dim_rows=5000, seed=4)
    p["p_price"][:] = 100_000
    p["p_discount"][:] = 0
    p["p_fk"][:] = (np.arange(p["p_fk"].shape[0]) % 5000 + 1).astype(np.int32)
    ctx.upload_table("dim", d)
    ctx.upload_table("probe", p)
    res, _ = ctx.run("template=join_topk;k=10;ship_gt=0;od_lt=3000")
    assert res.rows == O.join_topk(d, p, k=10, ship_gt=0, od_lt=3000)[0]


def test_join_topk_learned_size_overflow_is_reported(ctx):
    load_join(ctx, 200_000, 800_000)
    with pytest.raises(GpudbError) as e:
        ctx.run("template=join_topk;groups=4", "split=0")
    assert e.value.status == -7
    assert e.value.timing.device_error & DEVERR_HASH_OVERFLOW


def test_enqueue_pipelines_runs_and_reports_errors_at_sync(ctx):
    """Enqueued executions run back to back without a host wait; a device
    error raised by one of them survives later clean runs until sync()
    reads it, and sync() clears it."""
    d, p = load_join(ctx, 200_000, 800_000)
    top = O.join_topk(d, p, k=10)[0]
    ctx.set_use_graphs(True)
    try:
        for tune in ("", "split=1;stages=2;occ=3", "split=0"):
            q = ctx.prepare("template=join_topk", tune)
            for _ in range(5):
                ctx.enqueue(q)
            ctx.sync()
            res, t = ctx.run(q)
            assert res.rows == top and t.device_error == 0
        bad = ctx.prepare("template=join_topk;groups=4", "split=0")
        ok = ctx.prepare("template=join_topk", "split=1")
        ctx.enqueue(bad)
        ctx.enqueue(ok)
        with pytest.raises(GpudbError) as e:
            ctx.sync()
        assert e.value.status == -7 and e.value.device_error & DEVERR_HASH_OVERFLOW
        ctx.sync()
        res, t = ctx.run(ok)
        assert res.rows == top and t.device_error == 0
    finally:
        ctx.set_use_graphs(False)


def test_max_key_pass(ctx):
    d, _ = load_join(ctx, 123_457, 1000)
    assert ctx.register_max_key("b_key") == O.max_i32(d["b_key"]) == 123_457


def test_join_late_columns_read_in_place_from_host(ctx):
    """Late-materialised columns left in pinned host memory (zero-copy) give
    the same answer; a host column every row would read is refused before
    any launch."""
    import ctypes as C
    from gpudbmetalcodegen_b200 import _lib
    lib = _lib.load()
    d, p = load_join(ctx, 200_000, 800_000, seed=21)
    top, _, _ = O.join_topk(d, p, k=10)
    held = []
    for c in ("p_price", "p_discount", "p_fk"):
        a = p[c]
        ptr = lib.gpudb_host_alloc(a.nbytes)
        np.ctypeslib.as_array((C.c_uint8 * a.nbytes).from_address(ptr))[:] = a.view(np.uint8)
        held.append(ptr)
    try:
        ctx.register_host_column("probe", "p_price", held[0], p["p_price"].shape[0], 8)
        ctx.register_host_column("probe", "p_discount", held[1], p["p_discount"].shape[0], 8)
        res, t = ctx.run("template=join_topk")
        assert t.device_error == 0 and res.rows == top
        ctx.register_host_column("probe", "p_fk", held[2], p["p_fk"].shape[0], 4)
        with pytest.raises(GpudbError):
            ctx.run("template=join_topk")
        with pytest.raises(GpudbError):  # pageable memory is not accepted
            ctx.register_host_column("probe", "p_fk", p["p_fk"].ctypes.data, p["p_fk"].shape[0], 4)
    finally:
        for c in ("p_price", "p_discount", "p_fk"):
            ctx.upload_column("probe", c, p[c])
        ctx.synchronize()
        for ptr in held:
            lib.gpudb_host_free(C.c_void_p(ptr))


def test_join_topk_full_size(ctx):
    d, p = load_join(ctx, W.DIM_ROWS, W.PROBE_ROWS, seed=W.SEED)
    top, groups, distinct = O.join_topk(d, p, k=10)
    res, _ = ctx.run("template=join_topk")
    assert res.rows == top
    assert int(ctx.read_buffer("jg_nslots", np.uint64, 1)[0]) == groups
    assert int(ctx.read_buffer("jb_distinct", np.uint64, 1)[0]) == distinct
    res, _ = ctx.run("template=join_topk", "split=0")
    assert res.rows == top
    assert ctx.get_symbol("jt_groups") == distinct


# ---------------------------------------------------------------------------
# skewed group-by and hash join
# ---------------------------------------------------------------------------
GB_TUNES = ["", "layout=bucket8", "smem=10", "smem=12;layout=bucket8", "warp=0", "scan=direct;warp=0;smem=0",
            "vec=4", "vec=2;smem=0", "layout=packed", "layout=packed;smem=8;warp=0", "layout=packed;smem=0;warp=1",
            "smem=8;sprobe=4;warp=0", "sprobe=1",
            # the L2-resident warm tier: small (most keys spill past it), its
            # own probe lengths, the packed layout, no shared table
            "smem=8;warp=0;warm=8;wprobe=2", "smem=8;sprobe=4;warp=0;warm=14", "layout=packed;warm=12",
            "smem=0;warp=1;warm=16;wprobe=8"]


@pytest.fixture(scope="module")
def zipf_small():
    nkeys = 1 << 16
    return W.gen_zbuild(nkeys, seed=2), W.gen_zprobe(1_000_000, nkeys=nkeys, s=1.1, seed=2), nkeys


@pytest.mark.parametrize("tune", GB_TUNES)
def test_groupby_parity(ctx, zipf_small, tune):
    _, zp, nkeys = zipf_small
    ctx.upload_table("zprobe", zp)
    ctx.register_symbol("zgroups", nkeys)
    res, t = ctx.run("template=groupby", tune)
    assert t.device_error == 0
    k, c, s = O.groupby(zp["z_key"], zp["z_value"], cap=nkeys)
    assert np.array_equal(np.array(res.column("key")), k)
    assert np.array_equal(np.array(res.column("count")), c)
    assert np.array_equal(np.array(res.column("sum")), s)


@pytest.mark.parametrize("tune", ["", "layout=bucket8", "smem=11", "warp=0", "smem=8;sprobe=1", "sprobe=16"])
def test_hashjoin_parity(ctx, zipf_small, tune):
    zb, zp, _ = zipf_small
    ctx.upload_table("zbuild", zb)
    ctx.upload_table("zprobe", zp)
    res, _ = ctx.run("template=hashjoin", tune)
    k, c, s = O.hashjoin(zb, zp["z_key"], cap=zb["zb_key"].shape[0])
    assert np.array_equal(np.array(res.column("key")), k)
    assert np.array_equal(np.array(res.column("count")), c)
    assert np.array_equal(np.array(res.column("sum")), s)


# ---------------------------------------------------------------------------
# mixed-workload templates
# ---------------------------------------------------------------------------
@pytest.fixture(scope="module")
def mix_small():
    return W.gen_mix(400_000, nranks=1 << 20, dim_rows=50_000, seed=8), W.gen_mixdim(50_000, seed=8)


@pytest.mark.parametrize("thr", [100, 5000, 9900])
def test_mix_templates_parity(ctx, mix_small, thr):
    m, md = mix_small
    ctx.upload_table("mix", m)
    ctx.upload_table("mixdim", md)
    res, _ = ctx.run(f"template=mix_agg;thr={thr}")
    assert res.rows == [O.mix_agg(m, thr)]
    res, _ = ctx.run(f"template=mix_join;thr={thr};attr_lt=400")
    assert res.rows == [O.mix_join(md, m, 400, thr)]
    for key_col, card in (("m_rank_u", 1000), ("m_rank_z", 50_000)):
        ctx.register_symbol("mix_groups", card)
        res, _ = ctx.run(f"template=mix_groupby;thr={thr};card={card};key={key_col}")
        k, c, s = O.mix_groupby(m, key_col, thr, card)
        assert np.array_equal(np.array(res.column("key")), k)
        assert np.array_equal(np.array(res.column("sum")), s)
        res, _ = ctx.run(f"template=mix_topk;thr={thr};card={card};key={key_col};k=7")
        assert res.rows == O.topk(k, s, 7)


def test_autotuner_never_changes_an_answer(ctx, tmp_path):
    from gpudbmetalcodegen_b200 import autotune as A
    f = W.gen_fact(2_000_000, seed=19)
    ctx.upload_table("fact", f)
    cache = A.TuneCache(tmp_path / "dev.json")
    log = []
    space = {"bs": ["512", "256"], "tile": ["0", "1024"], "stages": ["4", "2"], "keyed": ["0", "1", "4"]}
    tune, best, default = A.tune_query(ctx, "template=q1", ctx.largest_table_rows(), space=space, cache=cache,
                                       log=log, reps=3, rounds=1)
    assert best <= default and len(log) >= 4
    res, _ = ctx.run("template=q1", tune)
    assert_q1_equal(res, O.q1(f))
    assert cache.get("q1", ctx.largest_table_rows()) == tune
    ctx._tune_cache = cache
    assert ctx.prepare("template=q1", "auto").tune == tune


def test_collect_reads_the_last_graphed_replay(ctx):
    """Back-to-back graph replays enqueued without a host wait, then the
    result the last one left in the buffers is collected without running
    the plan again, and equals the oracle's (what the benchmark checks after
    its timed steps)."""
    d, p = load_join(ctx, 100_000, 400_000, seed=17)
    q = ctx.prepare("template=join_topk", "")
    ctx.set_use_graphs(True)
    try:
        for _ in range(6):
            ctx.enqueue(q)
        ctx.sync()
        res = ctx.collect(q)
    finally:
        ctx.set_use_graphs(False)
    assert res.rows == O.join_topk(d, p, k=10)[0]
