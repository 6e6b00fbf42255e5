"""GPU: the continuous-batching server. Every answer served in the mix of a
Poisson trace equals the same query run alone and the CPU oracle's answer
(bit-exact), at two offered rates, with overflow re-runs counted and the
HBM budget respected."""
import numpy as np
import pytest

from gpudbmetalcodegen_b200 import batch as B
from gpudbmetalcodegen_b200 import serve as S
from gpudbmetalcodegen_b200 import workloads as W
from mix_oracle import oracle_result

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup(ctx):
    tables = B.MixTables(rows=2_000_000, zipf_s=(1.1,), nranks=1 << 20, dim_rows=200_000, seed=31, host=True)
    log = B.ExecutionLog()
    B.log_executions(tables, W.gen_mixed_queries(4000, seed=7, table_rows=tables.rows, n_tables=1,
                                                 min_rows=10_000, max_rows=tables.rows, max_card=1 << 20), log)
    sizer, _ = B.train_sizer(log, seed=2, epochs=40, batch=256)
    plain = B.PlainRunner(ctx, tables)
    yield tables, sizer, plain
    sizer.close()


@pytest.mark.parametrize("rate", [500.0, 5000.0])
def test_served_results_equal_queries_alone(setup, rate):
    tables, sizer, plain = setup
    qs = W.gen_mixed_queries(120, seed=int(rate), table_rows=tables.rows, n_tables=1, min_rows=10_000,
                             max_rows=tables.rows, max_card=1 << 20)
    trace = S.poisson_trace(qs, rate=rate, seed=1)
    srv = S.Server(tables, sizer, plain=plain, workers=2, hbm_budget=150e9)
    served, rep = srv.serve(trace)
    srv.close()
    alone = [plain.run(q) for q in qs]
    bad = [(i, B.describe_difference(a, b)) for i, (a, b) in enumerate(zip(served, alone))
           if not B.same_result(a, b)]
    assert not bad, bad[:3]
    expect = [oracle_result(tables, q) for q in qs]
    bad = [(i, qs[i], B.describe_difference(a, b)) for i, (a, b) in enumerate(zip(served, expect))
           if not B.same_result(a, b)]
    assert not bad, bad[:3]
    s = rep.summary()
    assert s["requests"] == len(qs) and sum(rep.batch_sizes) == len(qs)
    assert np.all(rep.latencies_s > 0)
    assert s["p99_ms"] >= s["p50_ms"] > 0
    # the same trace with answers handed over as they complete
    fps = {}
    srv = S.Server(tables, sizer, plain=plain, workers=2, hbm_budget=150e9)
    _, rep2 = srv.serve(trace, on_result=lambda i, r: fps.__setitem__(i, B.result_fingerprint(r)))
    srv.close()
    assert [fps[i] for i in range(len(qs))] == [B.result_fingerprint(r) for r in alone]


def test_budget_too_small_is_an_error(setup):
    tables, sizer, plain = setup
    q = B.MixQuery("groupby", 0, 0, tables.rows, 9000, card=1 << 20)
    srv = S.Server(tables, sizer, plain=plain, workers=1, hbm_budget=tables.bytes() + 1_000_000)
    with pytest.raises(MemoryError):
        srv.serve([S.Request(0, q, 0.001)])
    srv.close()
