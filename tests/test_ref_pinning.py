"""Pinning the oracle to the reference engine itself.

tests/golden/ref_pinning.json holds outputs of the reference's own generated
kernels (its plan builder + operator emitters + codegen, compiled from the
reference tree and executed on the CPU by oracle/ref_harness; regenerate
with tests/golden/make_golden.py) for seeded inputs of this repo's
generator. The oracle must reproduce them: counts and integer-scaled sums
exactly where the reference's float arithmetic is exact, all other sums
within the reference's own golden-check tolerance (abs 1e-2 + rel 1e-4 in
currency units, codegen/codegen_main.cpp:47-48); group sets and order
exactly. When the harness is built on this host (oracle/_ref), the same
comparison also runs live on fresh seeds.
"""
import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "oracle" / "ref_harness"))

from gpudbmetalcodegen_b200 import workloads as W  # noqa: E402
from oracle import oracle_py as O  # noqa: E402

GOLDEN = json.loads((ROOT / "tests" / "golden" / "ref_pinning.json").read_text())
ABS, REL = 1e-2, 1e-4
FLAGS = {0: ("A", "F"), 1: ("A", "O"), 2: ("N", "F"), 3: ("N", "O"), 4: ("R", "F"), 5: ("R", "O")}


def close(a, b):
    return abs(a - b) <= ABS + REL * max(abs(a), abs(b))


def checksum(cols):
    return int(sum(int(np.asarray(a, dtype=np.int64).sum()) * (i + 1) for i, a in enumerate(cols)) % (1 << 61))


def cases(plan):
    return [c for c in GOLDEN["cases"] if c["plan"] == plan]


def check_q1(ref_rows, fact):
    exact = O.q1(fact)
    assert [FLAGS[r["bucket"]] for r in ref_rows] == [(e["flag_a"], e["flag_b"]) for e in exact]
    for r, e in zip(ref_rows, exact):
        assert r["count_order"] == e["count_order"]
        assert r["sum_qty"] == 100 * e["sum_qty"]              # (uint)(qty*100.0f) is exact
        assert r["sum_disc"] == 100 * e["sum_disc"]            # (uint)(d/100*10000) is exact here
        assert close(r["sum_base_price"] / 100, e["sum_base_price"] / 100)
        assert close(r["sum_disc_price"] / 100, e["sum_disc_price"] / 1e4)
        assert close(r["sum_charge"] / 100, e["sum_charge"] / 1e6)


@pytest.mark.parametrize("case", cases("Q1"), ids=lambda c: f"n{c['rows']}")
def test_oracle_matches_reference_q1(case):
    f = W.gen_fact(case["rows"], seed=case["seed"])
    assert checksum(f.values()) == case["input_checksum"], "generator drift"
    check_q1(case["ref"], f)


@pytest.mark.parametrize("case", cases("Q6"), ids=lambda c: f"n{c['rows']}")
def test_oracle_matches_reference_q6(case):
    f = W.gen_fact(case["rows"], seed=case["seed"])
    assert checksum(f.values()) == case["input_checksum"]
    assert close(case["ref"]["revenue"] / 100, O.q6(f) / 1e4)


def join_groups_exact(d, p):
    keep = (d["b_segment"] == 1) & (d["b_order_day"] < 1170)
    qual = np.zeros(int(d["b_key"].max()) + 2, dtype=bool)
    qual[d["b_key"][keep]] = True
    m = (p["p_ship_day"] > 1170) & qual[p["p_fk"]]
    keys, inv = np.unique(p["p_fk"][m], return_inverse=True)
    sums = np.zeros(keys.shape[0], np.int64)
    np.add.at(sums, inv, p["p_price"][m] * (100 - p["p_discount"][m]))
    return keys, sums


def check_join(ref, d, p):
    keys, sums = join_groups_exact(d, p)
    assert list(keys) == ref["keys"]
    for s, r in zip(sums, ref["revenue"]):
        assert close(r, s / 1e4)
    # the oracle's top-k agrees with the reference's per-key revenue ranking
    top, groups, _ = O.join_topk(d, p, k=10)
    assert groups == len(ref["keys"])
    ranked = sorted(zip(ref["revenue"], ref["keys"]), key=lambda x: (-x[0], x[1]))[:10]
    assert [k for _, k in ranked] == [k for k, _ in top]


@pytest.mark.parametrize("case", cases("JOIN"), ids=lambda c: f"p{c['probe_rows']}")
def test_oracle_matches_reference_join(case):
    d = W.gen_dim(case["dim_rows"], seed=case["seed"])
    p = W.gen_probe(case["probe_rows"], dim_rows=case["dim_rows"], seed=case["seed"])
    assert checksum(list(d.values()) + list(p.values())) == case["input_checksum"]
    check_join(case["ref"], d, p)


def check_join_rows(ref, d, p):
    """The reference's materialised join rows: the same (row, key) pairs as
    the oracle, its float revenue within the golden tolerance of the exact
    one (1e-4 currency units)."""
    exp = O.join_rows(d, p)
    assert ref["row"] == [r for r, _, _ in exp]
    assert ref["key"] == [k for _, k, _ in exp]
    for a, (_, _, v) in zip(ref["revenue"], exp):
        assert close(a, v / 1e4)


@pytest.mark.parametrize("case", cases("JOINROWS"), ids=lambda c: f"p{c['probe_rows']}")
def test_oracle_matches_reference_join_rows(case):
    d = W.gen_dim(case["dim_rows"], seed=case["seed"])
    p = W.gen_probe(case["probe_rows"], dim_rows=case["dim_rows"], seed=case["seed"])
    assert checksum(list(d.values()) + list(p.values())) == case["input_checksum"]
    assert len(case["ref"]["row"]) > 100
    check_join_rows(case["ref"], d, p)


def check_groupby(ref, m, thr, card):
    k, c, s = O.mix_groupby(m, "m_rank_u", thr, card)
    assert list(k) == ref["keys"]
    assert list(c) == ref["count"]
    for a, b in zip(s, ref["sum"]):
        assert close(float(a), b)


@pytest.mark.parametrize("case", cases("GROUPBY"), ids=lambda c: f"n{c['rows']}")
def test_oracle_matches_reference_groupby(case):
    m = W.gen_mix(case["rows"], nranks=1 << 20, dim_rows=1000, seed=case["seed"])
    assert checksum([m["m_rank_u"], m["m_filter"], m["m_value"]]) == case["input_checksum"]
    check_groupby(case["ref"], m, case["thr"], case["card"])


def join_case(case):
    d = W.gen_dim(case["dim_rows"], seed=case["seed"])
    p = W.gen_probe(case["probe_rows"], dim_rows=case["dim_rows"], seed=case["seed"])
    assert checksum(list(d.values()) + list(p.values())) == case["input_checksum"]
    return d, p


def check_anti(ref, d, p):
    """The reference's anti-join (BitmapBuild, AntiBitmapProbe, per-discount
    AtomicCount and float AtomicAgg of the price): the same non-empty bins
    and counts as the oracle, the float price sums within the golden
    tolerance of the exact cent sums."""
    exp = O.anti_join(d, p)
    assert ref["bin"] == [b for b, _, _ in exp]
    assert ref["count"] == [c for _, c, _ in exp]
    for a, (_, _, s) in zip(ref["sum_price"], exp):
        assert close(a, s / 100)


@pytest.mark.parametrize("case", cases("ANTI"), ids=lambda c: f"p{c['probe_rows']}")
def test_oracle_matches_reference_anti(case):
    check_anti(case["ref"], *join_case(case))


@pytest.mark.parametrize("case", cases("HIST"), ids=lambda c: f"p{c['probe_rows']}")
def test_oracle_matches_reference_histogram(case):
    """The reference's count histogram (AtomicCount per key, ArrayLookup of
    each build key's count, AtomicCount into bins): exact."""
    d, p = join_case(case)
    exp = O.histogram(d, p)
    assert case["ref"]["bin"] == [c for c, _ in exp]
    assert case["ref"]["keys"] == [k for _, k in exp]


@pytest.mark.parametrize("case", cases("DIRECT"), ids=lambda c: f"p{c['probe_rows']}")
def test_oracle_matches_reference_direct(case):
    """The reference's direct-address join (ArrayStore of the qualifying build
    keys' order day, ArrayLookup per probe row, float AtomicAgg per key)
    yields the hash join's groups and revenues."""
    check_join(case["ref"], *join_case(case))


def check_multi_join(ref, snow):
    """The reference's Q5 plan (nation bitmap, customer / supplier / orders
    nation maps, same-nation probe with float AtomicAgg per nation): the
    oracle's nations, its exact revenues within the golden tolerance."""
    exp = O.multi_join(snow)
    assert ref["nation"] == [n for n, _ in exp]
    for a, (_, v) in zip(ref["revenue"], exp):
        assert close(a, v / 1e4)


@pytest.mark.parametrize("case", cases("Q5"), ids=lambda c: f"l{c['sizes'][3]}")
def test_oracle_matches_reference_multi_join(case):
    snow = W.gen_snowflake(*case["sizes"], seed=case["seed"])
    assert checksum([a for t in snow.values() for a in t.values()]) == case["input_checksum"]
    assert len(case["ref"]["nation"]) == 5
    check_multi_join(case["ref"], snow)


# ---------------------------------------------------------------------------
# live: the reference's kernels on fresh seeds (only where the harness exists)
# ---------------------------------------------------------------------------
def _live():
    try:
        import ref_run
    except ImportError:
        return None
    return ref_run if ref_run.available() else None


@pytest.mark.skipif(_live() is None, reason="reference harness not built on this host")
def test_live_reference_matches_oracle():
    R = _live()
    rk = R.RefKernels()
    for n, seed in ((7_777, 101), (33_001, 202)):
        f = W.gen_fact(n, seed=seed)
        check_q1(rk.keyed("Q1", rk.run("Q1", R.fact_as_reference(f), {"lineitem": n}, {})), f)
        ref6 = rk.scalar("Q6", rk.run("Q6", R.fact_as_reference(f), {"lineitem": n}, {}))
        assert close(ref6["revenue"] / 100, O.q6(f) / 1e4)
    nd, npr = 20_000, 90_000
    d = W.gen_dim(nd, seed=303)
    p = W.gen_probe(npr, dim_rows=nd, seed=303)
    cols = {"b_key": d["b_key"], "b_order_day": d["b_order_day"], "b_segment": d["b_segment"].view(np.int8),
            "p_fk": p["p_fk"], "p_ship_day": p["p_ship_day"], "p_price": (p["p_price"] / 100.0).astype(np.float32),
            "p_discount": (p["p_discount"] / 100.0).astype(np.float32)}
    b = rk.run("JOIN", cols, {"dim": nd, "probe": npr}, {"maxKey": int(d["b_key"].max()) + 1})
    keys = np.nonzero(b["d_revenue"] > 0)[0]
    check_join({"keys": [int(k) for k in keys], "revenue": [float(b["d_revenue"][k]) for k in keys]}, d, p)
    b = rk.run("JOINROWS", cols, {"dim": nd, "probe": npr}, {"maxKey": int(d["b_key"].max()) + 1})
    n = int(b["d_jr_n"][0])
    rows = sorted(zip(b["d_jr_row"][:n].tolist(), b["d_jr_key"][:n].tolist(), b["d_jr_rev"][:n].tolist()))
    check_join_rows({"row": [r for r, _, _ in rows], "key": [k for _, k, _ in rows],
                     "revenue": [float(v) for _, _, v in rows]}, d, p)
    b = rk.run("DIRECT", cols, {"dim": nd, "probe": npr}, {"maxKey": int(d["b_key"].max()) + 1})
    keys = np.nonzero(b["d_d_rev"] > 0)[0]
    check_join({"keys": [int(k) for k in keys], "revenue": [float(b["d_d_rev"][k]) for k in keys]}, d, p)
    b = rk.run("ANTI", dict(cols, p_discount=p["p_discount"].astype(np.int32)), {"dim": nd, "probe": npr},
               {"maxKey": int(d["b_key"].max()) + 1})
    bins = [k for k in range(11) if b["d_a_cnt"][k]]
    check_anti({"bin": bins, "count": [int(b["d_a_cnt"][k]) for k in bins],
                "sum_price": [float(b["d_a_sum"][k]) for k in bins]}, d, p)
    b = rk.run("HIST", {"p_fk": p["p_fk"], "p_ship_day": p["p_ship_day"], "b_key": d["b_key"]},
               {"dim": nd, "probe": npr}, {"maxKey": int(d["b_key"].max()) + 1})
    assert [(c, int(b["d_h_hist"][c])) for c in range(256) if b["d_h_hist"][c]] == O.histogram(d, p)
    snow = W.gen_snowflake(2_000, 150, 20_000, 90_000, seed=505)
    cols, rows, syms = R.snow_as_reference(snow)
    rev = rk.run("Q5", cols, rows, syms, scalars={"asia_rk": 2})["d_nation_revenue"]
    check_multi_join({"nation": [n for n in range(25) if rev[n]], "revenue": [float(v) for v in rev if v]}, snow)
    m = W.gen_mix(40_000, nranks=1 << 20, dim_rows=1000, seed=404)
    cols = {"m_rank_u": m["m_rank_u"], "m_filter": m["m_filter"], "m_value": m["m_value"].astype(np.float32)}
    b = rk.run("GROUPBY", cols, {"mix": 40_000}, {"card": 500}, scalars={"thr": 7000, "card": 500})
    keys = np.nonzero(b["d_cnt"])[0]
    check_groupby({"keys": [int(k) for k in keys], "count": [int(b["d_cnt"][k]) for k in keys],
                   "sum": [float(b["d_sum"][k]) for k in keys]}, m, 7000, 500)
