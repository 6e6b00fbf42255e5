"""Oracle known-answer tests on hand-computed tiny tables, and properties of
the seeded generators (CPU only)."""
import numpy as np
import pytest

from gpudbmetalcodegen_b200 import workloads as W
from oracle import oracle_py as O


def tiny_fact(rows):
    cols = {k: np.array([r[i] for r in rows], dtype=v) for i, (k, v) in enumerate(W.FACT_COLUMNS.items())}
    return cols


def test_q1_known_answer_buckets_filter_and_empty_groups():
    A, N, R, F, Os = ord("A"), ord("N"), ord("R"), ord("F"), ord("O")
    # ship, qty, price, disc, tax, flag_a, flag_b
    fact = tiny_fact([
        (10, 5, 100000, 4, 2, A, F),
        (20, 7, 200000, 0, 8, A, F),
        (3000, 9, 999999, 1, 1, A, F),   # filtered out by ship_day <= 2436
        (2436, 1, 90000, 10, 0, N, Os),  # boundary row kept
        (5, 2, 150000, 5, 3, R, F),
    ])
    rows = O.q1(fact, ship_le=2436)
    assert [(r["flag_a"], r["flag_b"]) for r in rows] == [("A", "F"), ("N", "O"), ("R", "F")]
    af = rows[0]
    assert af["sum_qty"] == 12 and af["count_order"] == 2
    assert af["sum_base_price"] == 300000
    assert af["sum_disc_price"] == 100000 * 96 + 200000 * 100
    assert af["sum_charge"] == 100000 * 96 * 102 + 200000 * 100 * 108
    assert af["sum_disc"] == 4
    assert af["avg_qty"] == 6.0 and af["avg_price"] == 150000.0
    no = rows[1]
    assert no["sum_disc_price"] == 90000 * 90 and no["sum_charge"] == 90000 * 90 * 100


def test_q1_sum_charge_needs_128_bits():
    n = 100
    fact = tiny_fact([(0, 50, 10_500_000, 0, 8, ord("A"), ord("F"))] * n)
    # scale one row's price so the per-group total exceeds int64
    big = 10_500_000
    rows = O.q1(fact)
    assert rows[0]["sum_charge"] == n * big * 100 * 108
    # 128-bit path: replicate to force > 2^63 in the exact sum
    fact = {k: np.tile(v, 900_000) for k, v in fact.items()}
    rows = O.q1(fact)
    total = 90_000_000 * big * 100 * 108
    assert total > 2**63 and rows[0]["sum_charge"] == total


def test_q6_known_answer():
    fact = tiny_fact([
        (400, 10, 100000, 6, 0, 65, 70),   # kept
        (400, 24, 100000, 6, 0, 65, 70),   # qty not < 24
        (364, 10, 100000, 6, 0, 65, 70),   # day out of range
        (729, 1, 300000, 5, 0, 65, 70),    # kept (day boundary, disc low edge)
        (730, 1, 300000, 7, 0, 65, 70),    # day == lt excluded
        (500, 2, 50000, 7, 0, 65, 70),     # kept (disc high edge)
        (500, 2, 50000, 8, 0, 65, 70),     # disc out of range
    ])
    assert O.q6(fact) == 100000 * 6 + 300000 * 5 + 50000 * 7


def test_join_topk_known_answer_with_ties():
    dim = {"b_key": np.array([3, 1, 2, 5, 4], np.int32), "b_order_day": np.array([100, 100, 2000, 100, 100], np.int32),
           "b_segment": np.array([1, 1, 1, 0, 1], np.uint8)}
    # qualifying build keys: 3, 1, 4 (key 2 fails order_day, key 5 fails segment)
    probe = {"p_fk": np.array([3, 1, 1, 4, 2, 5, 3, 4], np.int32),
             "p_ship_day": np.array([2000, 2000, 2000, 2000, 2000, 2000, 10, 2000], np.int32),
             "p_price": np.array([100, 50, 50, 100, 999, 999, 999, 0], np.int64),
             "p_discount": np.array([0, 0, 0, 0, 0, 0, 0, 0], np.int64)}
    top, groups, distinct = O.join_topk(dim, probe, k=10)
    assert distinct == 3
    assert groups == 3
    # sums: key1 = 10000, key3 = 10000 (row with ship 10 filtered), key4 = 10000 + 0
    assert top == [(1, 10000), (3, 10000), (4, 10000)]  # all tie -> ascending key
    top2, _, _ = O.join_topk(dim, probe, k=2)
    assert top2 == [(1, 10000), (3, 10000)]


def test_join_rows_known_answer_agrees_with_join_topk():
    dim = {"b_key": np.array([3, 1, 2, 5, 4], np.int32), "b_order_day": np.array([100, 100, 2000, 100, 100], np.int32),
           "b_segment": np.array([1, 1, 1, 0, 1], np.uint8)}
    probe = {"p_fk": np.array([3, 1, 1, 4, 2, 5, 3, 4], np.int32),
             "p_ship_day": np.array([2000, 2000, 2000, 2000, 2000, 2000, 10, 2000], np.int32),
             "p_price": np.array([100, 50, 50, 100, 999, 999, 999, 0], np.int64),
             "p_discount": np.array([0, 0, 0, 0, 0, 0, 0, 10], np.int64)}
    rows = O.join_rows(dim, probe)
    # rows 4 (key 2) and 5 (key 5) have no qualifying build key; row 6 ships too early
    assert rows == [(0, 3, 10000), (1, 1, 5000), (2, 1, 5000), (3, 4, 10000), (7, 4, 0)]
    # grouping the materialised rows gives the aggregate pipeline's answer
    sums = {}
    for _, k, v in rows:
        sums[k] = sums.get(k, 0) + v
    top, _, _ = O.join_topk(dim, probe, k=10)
    assert sorted(sums.items(), key=lambda kv: (-kv[1], kv[0])) == top
    assert O.join_rows(dim, probe, od_lt=0) == []


def _tiny_join():
    dim = {"b_key": np.array([3, 1, 2, 5, 4], np.int32), "b_order_day": np.array([100, 100, 2000, 100, 100], np.int32),
           "b_segment": np.array([1, 1, 1, 0, 1], np.uint8)}
    probe = {"p_fk": np.array([3, 1, 1, 4, 2, 5, 3, 4, 9], np.int32),
             "p_ship_day": np.array([2000, 2000, 2000, 2000, 2000, 2000, 10, 2000, 2000], np.int32),
             "p_price": np.array([100, 50, 50, 100, 999, 998, 997, 0, 7], np.int64),
             "p_discount": np.array([0, 0, 0, 0, 3, 3, 0, 10, 3], np.int64)}
    return dim, probe


def test_join_direct_known_answer_carries_the_build_attributes():
    dim, probe = _tiny_join()
    dim["b_order_day"] = np.array([100, 101, 2000, 100, 104], np.int32)
    # the join's top k with the matched build row's order_day and segment
    assert O.join_direct(dim, probe, k=10) == [(1, 10000, 101, 1), (3, 10000, 100, 1), (4, 10000, 104, 1)]
    assert O.join_direct(dim, probe, od_lt=0) == []


def test_anti_join_known_answer():
    dim, probe = _tiny_join()
    # qualifying keys 3, 1, 4; anti-probe keeps rows with keys 2, 5 and 9
    # (9 lies beyond every build key, so it is absent from the bitmap);
    # row 6 ships too early
    assert O.anti_join(dim, probe) == [(3, 3, 999 + 998 + 7)]
    # with no qualifying key every shipped row passes
    assert O.anti_join(dim, probe, od_lt=0) == [(0, 4, 100 + 50 + 50 + 100), (3, 3, 999 + 998 + 7), (10, 1, 0)]
    bad = dict(probe, p_discount=np.array([0, 0, 0, 0, 11, 3, 0, 10, 3], np.int64))
    with pytest.raises(ValueError):
        O.anti_join(dim, bad)


def test_histogram_known_answer():
    dim, probe = _tiny_join()
    probe = {k: v[:8] for k, v in probe.items()}  # drop the key beyond the build keys
    # shipped rows per key: 1 -> 2, 2 -> 1, 3 -> 1 (one row ships too early), 4 -> 2, 5 -> 1
    assert O.histogram(dim, probe) == [(1, 3), (2, 2)]
    assert O.histogram(dim, probe, ship_gt=5000) == [(0, 5)]
    with pytest.raises(ValueError):
        O.histogram(dim, probe, nbins=2)  # a count of 2 needs three bins
    with pytest.raises(ValueError):
        O.histogram(dim, _tiny_join()[1])  # key 9 has no slot


def test_new_chains_agree_with_numpy_restatements():
    """The C oracle of the anti-join and histogram chains against plain
    numpy restatements on seeded tables."""
    d = W.gen_dim(5000, seed=8)
    p = W.gen_probe(40000, dim_rows=5000, seed=8)
    keep = (d["b_segment"] == 1) & (d["b_order_day"] < 1170)
    qual = np.zeros(5002, bool)
    qual[d["b_key"][keep]] = True
    ok = (p["p_ship_day"] > 1170) & ~qual[p["p_fk"]]
    cnt = np.bincount(p["p_discount"][ok], minlength=11)
    sm = np.bincount(p["p_discount"][ok], weights=p["p_price"][ok].astype(np.float64), minlength=11)
    assert O.anti_join(d, p) == [(b, int(cnt[b]), int(sm[b])) for b in range(11) if cnt[b]]
    per_key = np.bincount(p["p_fk"][p["p_ship_day"] > 1170], minlength=5001)
    h = np.bincount(per_key[d["b_key"]], minlength=256)
    assert O.histogram(d, p) == [(c, int(h[c])) for c in range(256) if h[c]]


def test_groupby_and_hashjoin_known_answer():
    key = np.array([5, -3, 5, 9, -3, 5], np.int64)
    val = np.array([1, 2, 3, 4, 5, 6], np.int64)
    k, c, s = O.groupby(key, val, cap=16)
    assert list(k) == [-3, 5, 9] and list(c) == [2, 3, 1] and list(s) == [7, 10, 4]
    zb = {"zb_key": np.array([9, 5, 7], np.int64), "zb_payload": np.array([10, 20, 30], np.int32)}
    k, c, s = O.hashjoin(zb, key, cap=16)
    assert list(k) == [5, 9] and list(c) == [3, 1] and list(s) == [60, 10]


def test_topk_order_value_desc_key_asc():
    keys = np.array([7, 3, 9, 1, 4], np.int64)
    vals = np.array([5, 9, 9, 1, 5], np.int64)
    assert O.topk(keys, vals, 3) == [(3, 9), (9, 9), (4, 5)]


def test_generators_are_slice_reproducible():
    full = W.gen_fact(50_000, seed=7)
    part = W.gen_fact(10_000, seed=7, row0=20_000)
    for c in W.FACT_COLUMNS:
        assert np.array_equal(full[c][20_000:30_000], part[c])
    d_full = W.gen_dim(1000, seed=7)
    d_part = W.gen_dim(1000, seed=7, row0=100, count=50)
    assert np.array_equal(d_full["b_key"][100:150], d_part["b_key"])
    z1 = W.gen_zprobe(5000, nkeys=1 << 12, seed=3)
    z2 = W.gen_zprobe(1000, nkeys=1 << 12, seed=3, row0=2000)
    assert np.array_equal(z1["z_key"][2000:3000], z2["z_key"])


def test_fact_distributions_and_four_groups():
    f = W.gen_fact(200_000)
    assert f["f_ship_day"].min() >= 0 and f["f_ship_day"].max() <= 2526
    assert f["f_quantity"].min() >= 1 and f["f_quantity"].max() <= 50
    assert f["f_price"].min() >= 90_000 and f["f_price"].max() <= 10_500_000
    assert f["f_discount"].max() <= 10 and f["f_tax"].max() <= 8
    rows = O.q1(f)
    assert len(rows) == 4
    assert {(r["flag_a"], r["flag_b"]) for r in rows} == {("A", "F"), ("N", "F"), ("N", "O"), ("R", "F")}
    sel = (f["f_ship_day"] <= 2436).mean()
    assert 0.95 < sel < 0.97


def test_dim_keys_are_a_permutation_and_probe_follows_order_day():
    n = 100_000
    d = W.gen_dim(n)
    assert np.array_equal(np.sort(d["b_key"]), np.arange(1, n + 1, dtype=np.int32))
    p = W.gen_probe(50_000, dim_rows=n)
    od = np.empty(n + 1, np.int32)
    od[d["b_key"]] = d["b_order_day"]
    delta = p["p_ship_day"] - od[p["p_fk"]]
    assert delta.min() >= 1 and delta.max() <= 121


def test_zipf_top_key_share():
    z = W.gen_zprobe(2_000_000, nkeys=1 << 22, s=1.1)
    _, counts = np.unique(z["z_key"], return_counts=True)
    share = counts.max() / z["z_key"].shape[0]
    assert 0.11 < share < 0.128  # 1 / H_{2^22}(1.1) = 0.119
    zb = W.gen_zbuild(1 << 16)
    assert np.unique(zb["zb_key"]).shape[0] == 1 << 16
    assert not (zb["zb_key"] == -1).any()


def test_multi_join_known_answer():
    """Q5 shape on a hand-built snowflake: nations 2 and 7 are region 2."""
    nation = {"n_key": np.arange(25, dtype=np.int32), "n_region": (np.arange(25) % 5).astype(np.int32)}
    cust = {"c_key": np.array([1, 2, 3], np.int32), "c_nation": np.array([2, 7, 3], np.int32)}
    supp = {"s_key": np.array([1, 2, 3], np.int32), "s_nation": np.array([2, 7, 2], np.int32)}
    ords = {"o_key": np.array([1, 2, 3, 4], np.int32), "o_cust": np.array([1, 2, 3, 1], np.int32),
            "o_day": np.array([800, 800, 800, 5], np.int32)}
    # order 1 (cust nation 2), 2 (nation 7), 3 (nation 3, not in the region), 4 (too early)
    line = {"l_okey": np.array([1, 1, 2, 2, 3, 4], np.int32), "l_supp": np.array([1, 2, 2, 3, 1, 1], np.int32),
            "l_price": np.array([100, 200, 300, 400, 500, 600], np.int64),
            "l_discount": np.array([0, 0, 10, 0, 0, 0], np.int64)}
    snow = {"nation": nation, "cust": cust, "supp": supp, "ord": ords, "line": line}
    # line 0: order nation 2, supplier nation 2 -> 100 * 100; line 1: 2 vs 7 no;
    # line 2: 7 vs 7 -> 300 * 90; line 3: 7 vs 2 no; line 4: order not kept; line 5: too early
    assert O.multi_join(snow) == [(2, 10000), (7, 27000)]
    assert O.multi_join(snow, region=3) == []  # nation 3 is region 3, but suppliers are not
