"""Host-side logic of the serving loop (no GPU): the Poisson trace, the
admission cost bound, and the FIFO queue of the one-at-a-time baseline."""
import numpy as np
import pytest

from gpudbmetalcodegen_b200 import batch as B
from gpudbmetalcodegen_b200 import serve as S


def test_poisson_trace_rate_and_order():
    qs = [B.MixQuery("agg", 0, 0, 10, 5)] * 20000
    tr = S.poisson_trace(qs, rate=2000.0, seed=3)
    t = np.array([r.arrival for r in tr])
    assert np.all(np.diff(t) > 0)
    assert len(tr) / t[-1] == pytest.approx(2000.0, rel=0.03)
    gaps = np.diff(t)
    assert gaps.std() / gaps.mean() == pytest.approx(1.0, rel=0.05)  # exponential: cv = 1
    assert [r.id for r in tr] == list(range(len(tr)))


def test_admission_cost_bounds_the_table():
    g = B.MixQuery("groupby", 0, 0, rows=1_000_000, thr=5000, card=1 << 20)
    small = B.MixQuery("groupby", 0, 0, rows=100, thr=5000, card=1 << 20)
    # slots for min(card, rows) groups at load factor <= 1/2, 44 B per slot
    assert S.query_hbm_bytes(g, 0) == (1 << 21) * 44 + 4096
    assert S.query_hbm_bytes(small, 0) == 256 * 44 + 4096
    assert S.query_hbm_bytes(B.MixQuery("join", 0, 0, 10, 5), 30_000_000) == 30_000_000 // 8 + 4096
    assert S.query_hbm_bytes(B.MixQuery("agg", 0, 0, 10, 5), 0) == 4096


def test_fifo_queue_of_the_plain_baseline():
    qs = [B.MixQuery("agg", 0, 0, 10, 5)] * 4
    tr = [S.Request(i, q, a) for i, (q, a) in enumerate(zip(qs, [0.0, 0.1, 0.2, 1.0]))]
    service = np.array([0.15, 0.15, 0.15, 0.05])
    _, rep, _ = S.serve_plain(None, tr, service_s=service)
    # completions: 0.15, 0.30, 0.45, 1.05
    assert np.allclose(rep.latencies_s, [0.15, 0.20, 0.25, 0.05])
    s = rep.summary()
    assert s["requests"] == 4 and s["p50_ms"] == pytest.approx(175.0)


def test_live_plain_baseline_waits_for_arrivals_and_queues():
    import time

    class Slow:  # a plain path whose every query takes 30 ms
        def run(self, q):
            time.sleep(0.03)
            return ("scalar", 1, q.thr)

    qs = [B.MixQuery("agg", 0, 0, 10, t) for t in (1, 2, 3)]
    tr = [S.Request(i, q, a) for i, (q, a) in enumerate(zip(qs, [0.0, 0.01, 0.2]))]
    res, rep = S.serve_plain_live(Slow(), tr)
    assert [r[2] for r in res] == [1, 2, 3]  # arrival order
    lat = rep.latencies_s
    # the second request queues behind the first; the third arrives to an idle server
    assert 0.03 <= lat[0] < 0.06 and 0.05 <= lat[1] < 0.09 and 0.03 <= lat[2] < 0.06
