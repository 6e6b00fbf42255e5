"""Plan -> CUDA codegen -> NVRTC (sm_100a) compile, all without a GPU.

Mirrors the reference's structural expectations: one kernel per phase,
bindings per operator, result schema per terminal operator."""
import pytest

from gpudbmetalcodegen_b200 import engine
from gpudbmetalcodegen_b200._lib import GpudbError

SPECS = [
    "template=q1", "template=q6", "template=join_topk", "template=join_topk;groups=200000",
    "template=groupby", "template=hashjoin", "template=colmax;table=dim;col=b_key",
    "template=distinct;card=1000;thr=5000", "template=mix_agg;thr=5000", "template=mix_groupby;card=1000",
    "template=mix_topk;card=1000;k=5", "template=mix_join;attr_lt=300",
    "template=distinct;params=1;key=m_rank_z", "template=mix_agg;params=1", "template=mix_join;params=1",
    "template=mix_groupby;params=1;compact=1", "template=mix_topk;params=1;k=10", "template=join_direct",
    "template=anti_join", "template=histogram", "template=q6_selvec", "template=multi_join", "template=groupby_sorted",
]
TUNES = ["", "bs=256;scan=direct", "bs=512;scan=tma;tile=2048;stages=3", "bs=1024;scan=tma;tile=1024;stages=2",
         "layout=bucket8;smem=11", "keyed=2", "keyed=3;warp=0"]


@pytest.mark.parametrize("spec", SPECS)
def test_every_template_compiles_for_sm100a(spec):
    q = engine.Query(spec)
    assert "extern \"C\" __global__" in q.source
    assert "registers" in q.compile_log  # ptxas -v resource line per kernel
    assert "phase 0" in q.plan


@pytest.mark.parametrize("tune", TUNES)
def test_tune_variants_compile(tune):
    for spec in ("template=q1", "template=groupby", "template=join_topk"):
        if "bucket8" in tune and spec == "template=join_topk":
            continue  # int32 group keys use the linear layout
        q = engine.Query(spec, tune)
        assert "__launch_bounds__" in q.source


def test_q1_structure_matches_reference_plan():
    q = engine.Query("template=q1")
    src, plan = q.source, q.plan
    # reference Q1: one phase, KeyedAgg(6 buckets) <- Selection <- Scan(lineitem)
    assert plan.count("phase ") == 1 and "Q1_reduce" in plan
    assert "KeyedAgg(d_q1_aggs, 6 buckets, 6 aggs, registers-switch)" in plan
    assert "f_ship_day[i] <= 2436" in src
    # reference bucket expression (metal_plan_builder.cpp:335)
    assert "(f_flag_a[i] == 'A' ? 0 : (f_flag_a[i] == 'N' ? 2 : 4)) + (f_flag_b[i] == 'F' ? 0 : 1)" in src
    kernels = src.split("// === Phase", 1)[1]
    assert "gpudb_bulk_g2s_stream(" in kernels and "multicast" not in src


def test_tma_scan_is_default_and_direct_mode_has_no_bulk_copies():
    tma = engine.Query("template=q6").source
    direct = engine.Query("template=q6", "scan=direct").source
    assert "gpudb_bulk_g2s_stream(" in tma.split("// === Phase")[1]
    assert "gpudb_bulk_g2s_stream(" not in direct.split("// === Phase")[1]


def test_join_topk_three_phases_and_sizing_step():
    plan = engine.Query("template=join_topk", "split=0").plan
    assert "JT_build" in plan and "JT_probe_group" in plan and "JT_topk" in plan
    assert "sizing jt_groups after phase 1 from counter jb_distinct" in plan
    given = engine.Query("template=join_topk;groups=1000", "split=0").plan
    assert "from '1000'" in given


def test_split_join_sizes_its_group_table_on_the_device():
    q = engine.Query("template=join_topk")  # the split plan is the default
    phases = [ln.split()[2].rstrip(":") for ln in q.plan.splitlines() if ln.strip().startswith("phase ")]
    assert phases == ["JT_build", "JT_probe", "JT_init", "JT_group", "JT_topk"]
    assert "sizing jt_groups" not in q.plan  # no host round trip between the phases
    init = q.source.split("// === Phase 2: JT_init ===")[1].split("// === Phase 3")[0]
    group = q.source.split("// === Phase 3: JT_group ===")[1].split("// === Phase 4")[0]
    for body in (init, group):
        assert "gpudb_device_log2cap((unsigned long long)(min(__ldg(jm_n), __ldg(jb_distinct))), jg_log2max)" in body


def test_join_rows_materialises_the_matches():
    q = engine.Query("template=join_rows;ship_gt=1000")
    phases = [ln.split()[2].rstrip(":") for ln in q.plan.splitlines() if ln.strip().startswith("phase ")]
    assert phases == ["JR_build", "JR_probe"]
    assert "Materialize(3 columns)" in q.plan and "gpudb_warp_reserve(jr_n" in q.source
    assert "p_ship_day[i] > 1000" in q.source


def test_top_k_over_a_slot_list_is_warp_cooperative():
    src = engine.Query("template=join_topk", "split=1").source
    topk = src.split("// === Phase 4: JT_topk ===")[1]
    assert "gpudb_topk_warp_offer<10>(" in topk and "_tk_v[" not in topk  # no per-thread k-lists
    assert "jt_top_floor" in topk  # block floors prune the grid merge


def test_hash_join_counts_matches_and_multiplies():
    q = engine.Query("template=hashjoin")
    phases = [ln.split()[2].rstrip(":") for ln in q.plan.splitlines() if ln.strip().startswith("phase ")]
    assert phases == ["HJ_build", "HJ_probe_count", "HJ_sum"]
    probe = q.source.split("// === Phase 1: HJ_probe_count ===")[1].split("// === Phase 2")[0]
    assert "hj_payload" not in probe  # the probe reads no payload
    assert "hj_sum[_ak0] = (long long)((long long)hj_payload[s] * (long long)hj_count[s]);" in q.source


def test_packed_layout_is_for_group_by_tables():
    q = engine.Query("template=groupby", "layout=packed")
    assert "packed" in q.plan and "zg_slots" in q.source and "gpudb_htp_insert64(" in q.source
    with pytest.raises(GpudbError) as e:
        engine.Query("template=hashjoin", "layout=packed")
    assert "group-by tables only" in e.value.message


def test_spec_errors_are_reported():
    with pytest.raises(GpudbError) as e:
        engine.Query("template=nope")
    assert "unknown template" in e.value.message
    with pytest.raises(GpudbError) as e:
        engine.Query("template=q1;bogus=1")
    assert "unknown key" in e.value.message
    with pytest.raises(GpudbError):
        engine.Query("template=q1", "bs=100")


def test_compile_check_reports_errors_with_numbered_source():
    ok, log, _ = engine.compile_check("extern \"C\" __global__ void k() { this is not cuda; }")
    assert not ok
    assert "1: extern" in log


def test_compare_canonical_semantics():
    a = "k,v\n1,10.0000\n2,20.0000\n"
    assert engine.compare_canonical(a, a) == ""
    assert engine.compare_canonical(a, "k,v\n1,10.0001\n2,20.0000\n") == ""
    assert "row count" in engine.compare_canonical(a, "k,v\n1,10.0\n")
    assert engine.compare_canonical(a, "k,v\n1,11.0\n2,20.0\n").startswith("row 1")
    assert engine.compare_canonical("x,k,v\nq,1,10\n", "k,v\n1,10\n") == ""  # shared columns only


def test_launch_bound_constants_are_not_compiled_in():
    """params=1: one module per template whatever the constants; the
    constants are kernel arguments bound from symbols at launch."""
    q = engine.Query("template=mix_groupby;params=1;compact=1;key=m_rank_z")
    assert "mix_thr" in q.source and "gpudb_mod_i32(m_rank_z[i], _mix_div)" in q.source
    assert "ConstantScalar long long mix_card  [mix_card]" in q.plan
    with pytest.raises(GpudbError):
        engine.Query("template=mix_agg;params=1;thr=5")  # a constant and params=1 at once


def test_hash_fill_sizes_the_table():
    default = engine.Query("template=groupby").plan
    assert "pow2ceil(max(2 * (zgroups), 16))" in default
    low = engine.Query("template=groupby", "htf=100").plan
    assert "pow2ceil(max((zgroups) * 100 / 100, 16))" in low
    join = engine.Query("template=hashjoin", "htf=125").plan
    assert "(n_zbuild) * 125 / 100" in join
    with pytest.raises(GpudbError):
        engine.Query("template=groupby", "htf=50")


def test_warm_tier_adds_a_flush_phase():
    q = engine.Query("template=groupby", "smem=8;warm=16;wprobe=4")
    assert "GB_warm_flush: HashWarmFlush(zg, 65536 warm slots)" in q.plan
    assert "gpudb_ht_try_insert64(zg_wkeys, 16," in q.source
    assert "zg_wkeys  [65536]  fill=255" in q.plan
    with pytest.raises(GpudbError):
        engine.Query("template=groupby", "warm=4")


def _tiles(q):
    import re
    return {t: int(n) for t, n in re.findall(r"scan of (\w+): (\d+)-row tiles", q.source)}


def test_split_join_tiles_hold_whole_consumer_rounds():
    """The split join's automatic scan tiles are whole rounds of its consumer
    threads (the block minus the producer warp, times the rows each takes
    per round), so no warp takes an extra round per tile; a streaming
    reduction keeps its power-of-two tile, and an explicit tile is kept."""
    assert _tiles(engine.Query("template=join_topk", "bs=512;tile=0;split=1;bvec=4")) == {"dim": 1920, "probe": 1920}
    t = _tiles(engine.Query("template=join_topk", "bs=256;tile=0;split=1;bvec=2"))
    assert t["dim"] % (224 * 2) == 0 and t["probe"] % 224 == 0 and t["dim"] % 16 == 0
    assert _tiles(engine.Query("template=q6", "bs=256;tile=0")) == {"fact": 1024}
    assert _tiles(engine.Query("template=join_topk", "bs=512;tile=2048;split=1;bvec=4")) == {"dim": 2048, "probe": 2048}
    assert _tiles(engine.Query("template=join_topk", "bs=512;tile=0;split=0")) == {"dim": 2048, "probe": 2048}
