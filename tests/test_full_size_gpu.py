"""GPU parity at the configurations' stated sizes, through the C-ABI,
against the CPU oracle (bit-exact):

* the skewed-key group-by and hash join: 120M probe rows with Zipf(1.1)
  keys over 2^22 distinct int64 keys and a 2^22-row build side — tables of
  64-224 MB, larger than L2, where the layouts, the shared hot-key cache
  and the probe bounds behave differently from small cases — under the
  default tuning and the layout / cache variants;
* the batched mixed form: the benchmark's 256 seeded queries over four
  resident 120M-row tables (cardinalities up to 2^22), run batched with
  exact sizing and with a learned sizer that is deliberately wrong for
  some queries (their tables overflow and they re-run exactly); a seeded
  subset of 40 queries covering every template is checked against the
  oracle on slices regenerated on the host, and every query of the two
  batched runs agrees with the other.
"""
import numpy as np
import pytest

from gpudbmetalcodegen_b200 import batch as B
from gpudbmetalcodegen_b200 import workloads as W
from mix_oracle import oracle_result
from oracle import oracle_py as O

pytestmark = pytest.mark.gpu

ZKEYS = 1 << 22
ZROWS = 120_000_000


@pytest.fixture(scope="module")
def zipf_full():
    zb = W.gen_zbuild(ZKEYS, seed=W.SEED)
    zp = W.gen_zprobe(ZROWS, nkeys=ZKEYS, s=1.1, seed=W.SEED)
    gb = O.groupby(zp["z_key"], zp["z_value"], cap=ZKEYS)
    hj = O.hashjoin(zb, zp["z_key"], cap=ZKEYS)
    return zb, zp, gb, hj


def _same(res, expect):
    k, c, s = expect
    assert np.array_equal(np.array(res.column("key")), k)
    assert np.array_equal(np.array(res.column("count")), c)
    assert np.array_equal(np.array(res.column("sum")), s)


@pytest.mark.parametrize("tune", ["", "layout=bucket8", "layout=packed", "smem=0", "sprobe=4",
                                  "bs=256;stages=2;smem=8;sprobe=4;warp=0",
                                  "bs=256;stages=2;smem=8;sprobe=4;warp=0;warm=16"])
def test_groupby_full_size(ctx, zipf_full, tune):
    _, zp, gb, _ = zipf_full
    ctx.upload_table("zprobe", zp)
    ctx.register_symbol("zgroups", ZKEYS)
    res, t = ctx.run("template=groupby", tune)
    assert t.device_error == 0
    _same(res, gb)


@pytest.mark.parametrize("tune", ["", "layout=bucket8", "smem=0", "sprobe=4", "stages=2;smem=8;warp=0"])
def test_hashjoin_full_size(ctx, zipf_full, tune):
    zb, zp, _, hj = zipf_full
    ctx.upload_table("zbuild", zb)
    ctx.upload_table("zprobe", {"z_key": zp["z_key"]})
    res, t = ctx.run("template=hashjoin", tune)
    assert t.device_error == 0
    _same(res, hj)


def test_mixed_batch_full_size(ctx):
    import torch
    tables = B.MixTables(rows=W.MIX_TABLE_ROWS, zipf_s=W.MIX_ZIPF_S, nranks=W.MIX_NRANKS,
                         dim_rows=W.MIX_DIM_ROWS, seed=W.SEED)
    qs = W.gen_mixed_queries(256, seed=W.SEED, table_rows=tables.rows)
    assert max(q.card for q in qs if q.grouped) > 1 << 21
    plain = B.PlainRunner(ctx, tables)

    exact = B.BatchRunner(tables, sizing="exact", plain=plain)
    got_exact, rep = exact.run(qs)
    exact.close()
    assert rep.overflowed == []

    # a sizer that predicts one group for every fourth grouped query: those
    # tables overflow on the device and the queries re-run exactly
    class Wrong(B.BatchRunner):
        def size(self, queries, report):
            sizes = super().size(queries, report)
            return [1 if (q.grouped and i % 4 == 0) else s for i, (q, s) in enumerate(zip(queries, sizes))]

    wrong = Wrong(tables, sizing="bound", plain=plain)
    got_wrong, rep = wrong.run(qs)
    wrong.close()
    assert len(rep.overflowed) > 0
    assert all(qs[i].grouped for i in rep.overflowed)
    bad = [i for i, (a, b) in enumerate(zip(got_exact, got_wrong)) if not B.same_result(a, b)]
    assert not bad, bad[:3]

    # a seeded subset of 40 queries against the oracle: every template, and
    # overflowed-and-re-run queries among them
    rng = np.random.default_rng(12345)
    pick = set(int(i) for i in rng.choice(len(qs), 32, replace=False))
    for tmpl in B.TEMPLATES:
        pick.update([i for i, q in enumerate(qs) if q.tmpl == tmpl][:2])
    pick.update(rep.overflowed[:4])
    pick = sorted(pick)[:40] if len(pick) > 40 else sorted(pick)
    assert {qs[i].tmpl for i in pick} == set(B.TEMPLATES)
    assert any(i in rep.overflowed for i in pick)
    for i in pick:
        e = oracle_result(tables, qs[i])
        assert B.same_result(got_exact[i], e), (i, qs[i], B.describe_difference(got_exact[i], e))
        assert B.same_result(got_wrong[i], e), (i, qs[i], B.describe_difference(got_wrong[i], e))
    torch.cuda.synchronize()
