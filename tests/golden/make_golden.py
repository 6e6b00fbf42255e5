"""Generate tests/golden/ref_pinning.json from the reference engine's own
kernels (built by oracle/ref_harness/build_ref.py from the reference tree and
run on the CPU by oracle/ref_harness/ref_run.py).

Each case records the generator parameters of its seeded inputs, a checksum
of those inputs (to detect generator drift) and the reference's outputs,
decoded as the reference's result collector decodes them. Run in a container
that holds the reference tree:

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle" / "ref_harness"))

from gpudbmetalcodegen_b200 import workloads as W  # noqa: E402


def checksum(cols) -> int:
    return int(sum(int(np.asarray(a, dtype=np.int64).sum()) * (i + 1) for i, a in enumerate(cols)) % (1 << 61))


def join_inputs(nd, npr, seed):
    d = W.gen_dim(nd, seed=seed)
    p = W.gen_probe(npr, dim_rows=nd, seed=seed)
    return d, p


def main():
    import build_ref
    import ref_run as R
    build_ref.build()
    rk = R.RefKernels()
    out = {"source": "reference code generator (metal_plan_builder/metal_operators/metal_codegen_base), "
                     "kernels executed on the CPU via oracle/ref_harness", "cases": []}

    for n, seed in ((20_000, 3), (65_537, 17)):
        f = W.gen_fact(n, seed=seed)
        cs = checksum(f.values())
        b = rk.run("Q1", R.fact_as_reference(f), {"lineitem": n}, {})
        out["cases"].append({"plan": "Q1", "rows": n, "seed": seed, "input_checksum": cs, "ref": rk.keyed("Q1", b)})
        b = rk.run("Q6", R.fact_as_reference(f), {"lineitem": n}, {})
        out["cases"].append({"plan": "Q6", "rows": n, "seed": seed, "input_checksum": cs, "ref": rk.scalar("Q6", b)})

    nd, npr, seed = 50_000, 200_000, 4
    d, p = join_inputs(nd, npr, seed)
    cols = {"b_key": d["b_key"], "b_order_day": d["b_order_day"], "b_segment": d["b_segment"].view(np.int8),
            "p_fk": p["p_fk"], "p_ship_day": p["p_ship_day"], "p_price": (p["p_price"] / 100.0).astype(np.float32),
            "p_discount": (p["p_discount"] / 100.0).astype(np.float32)}
    b = rk.run("JOIN", cols, {"dim": nd, "probe": npr}, {"maxKey": int(d["b_key"].max()) + 1})
    rev = b["d_revenue"]
    keys = np.nonzero(rev > 0)[0]
    out["cases"].append({"plan": "JOIN", "dim_rows": nd, "probe_rows": npr, "seed": seed,
                         "input_checksum": checksum(list(d.values()) + list(p.values())),
                         "ref": {"keys": [int(k) for k in keys], "revenue": [float(rev[k]) for k in keys]}})

    b = rk.run("JOINROWS", cols, {"dim": nd, "probe": npr}, {"maxKey": int(d["b_key"].max()) + 1})
    cnt = int(b["d_jr_n"][0])
    rows = sorted(zip(b["d_jr_row"][:cnt].tolist(), b["d_jr_key"][:cnt].tolist(), b["d_jr_rev"][:cnt].tolist()))
    out["cases"].append({"plan": "JOINROWS", "dim_rows": nd, "probe_rows": npr, "seed": seed,
                         "input_checksum": checksum(list(d.values()) + list(p.values())),
                         "ref": {"row": [r for r, _, _ in rows], "key": [k for _, k, _ in rows],
                                 "revenue": [float(v) for _, _, v in rows]}})

    n, seed, thr, card = 100_000, 5, 5000, 1000
    m = W.gen_mix(n, nranks=1 << 20, dim_rows=1000, seed=seed)
    cols = {"m_rank_u": m["m_rank_u"], "m_filter": m["m_filter"], "m_value": m["m_value"].astype(np.float32)}
    b = rk.run("GROUPBY", cols, {"mix": n}, {"card": card}, scalars={"thr": thr, "card": card})
    keys = np.nonzero(b["d_cnt"])[0]
    out["cases"].append({"plan": "GROUPBY", "rows": n, "seed": seed, "thr": thr, "card": card,
                         "input_checksum": checksum([m["m_rank_u"], m["m_filter"], m["m_value"]]),
                         "ref": {"keys": [int(k) for k in keys], "count": [int(b["d_cnt"][k]) for k in keys],
                                 "sum": [float(b["d_sum"][k]) for k in keys]}})

    # the anti-join, the count histogram and the direct-address join: the
    # reference's AntiBitmapProbe / AtomicCount + ArrayLookup / ArrayStore +
    # ArrayLookup chains over the same seeded build and probe tables
    nd, npr, seed = 20_000, 80_000, 6
    d, p = join_inputs(nd, npr, seed)
    cs = checksum(list(d.values()) + list(p.values()))
    price = (p["p_price"] / 100.0).astype(np.float32)
    cols = {"b_key": d["b_key"], "b_order_day": d["b_order_day"], "b_segment": d["b_segment"].view(np.int8),
            "p_fk": p["p_fk"], "p_ship_day": p["p_ship_day"], "p_price": price,
            "p_discount": p["p_discount"].astype(np.int32)}
    b = rk.run("ANTI", cols, {"dim": nd, "probe": npr}, {"maxKey": int(d["b_key"].max()) + 1})
    bins = [k for k in range(11) if b["d_a_cnt"][k]]
    out["cases"].append({"plan": "ANTI", "dim_rows": nd, "probe_rows": npr, "seed": seed, "input_checksum": cs,
                         "ref": {"bin": bins, "count": [int(b["d_a_cnt"][k]) for k in bins],
                                 "sum_price": [float(b["d_a_sum"][k]) for k in bins]}})
    b = rk.run("HIST", {"p_fk": p["p_fk"], "p_ship_day": p["p_ship_day"], "b_key": d["b_key"]},
               {"dim": nd, "probe": npr}, {"maxKey": int(d["b_key"].max()) + 1})
    bins = [k for k in range(256) if b["d_h_hist"][k]]
    out["cases"].append({"plan": "HIST", "dim_rows": nd, "probe_rows": npr, "seed": seed, "input_checksum": cs,
                         "ref": {"bin": bins, "keys": [int(b["d_h_hist"][k]) for k in bins]}})
    cols["p_discount"] = (p["p_discount"] / 100.0).astype(np.float32)
    b = rk.run("DIRECT", cols, {"dim": nd, "probe": npr}, {"maxKey": int(d["b_key"].max()) + 1})
    rev = b["d_d_rev"]
    keys = np.nonzero(rev > 0)[0]
    out["cases"].append({"plan": "DIRECT", "dim_rows": nd, "probe_rows": npr, "seed": seed, "input_checksum": cs,
                         "ref": {"keys": [int(k) for k in keys], "revenue": [float(rev[k]) for k in keys]}})

    # the multi-join through the reference's own Q5 plan (buildMetalPlan by name)
    nc, ns, no, nl, seed = 3_000, 200, 30_000, 120_000, 8
    snow = W.gen_snowflake(nc, ns, no, nl, seed=seed)
    cols, rows, syms = R.snow_as_reference(snow)
    b = rk.run("Q5", cols, rows, syms, scalars={"asia_rk": 2})
    rev = b["d_nation_revenue"]
    nations = [n for n in range(25) if rev[n]]
    out["cases"].append({"plan": "Q5", "sizes": [nc, ns, no, nl], "seed": seed,
                         "input_checksum": checksum([a for t in snow.values() for a in t.values()]),
                         "ref": {"nation": nations, "revenue": [float(rev[n]) for n in nations]}})

    path = Path(__file__).resolve().parent / "ref_pinning.json"
    path.write_text(json.dumps(out, separators=(",", ":")) + "\n")
    print(f"wrote {path} ({path.stat().st_size} bytes, {len(out['cases'])} cases)")


if __name__ == "__main__":
    main()
