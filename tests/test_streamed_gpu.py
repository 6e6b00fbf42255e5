"""Chunked streaming runs (gpudb_query_run_streamed) against the oracle:
the probe side of the join and the fact table of Q1 / Q6 streamed from
pinned host memory in ragged chunks, copied per chunk or read in place,
through the same generated kernels as the resident runs."""
import ctypes as C

import numpy as np
import pytest

from gpudbmetalcodegen_b200 import _lib
from gpudbmetalcodegen_b200 import workloads as W
from gpudbmetalcodegen_b200._lib import GpudbError
from oracle import oracle_py as O
from test_gpu_parity import assert_q1_equal

pytestmark = pytest.mark.gpu


class Pinned:
    """Pinned host copies of numpy columns, freed on exit."""

    def __init__(self):
        self.lib = _lib.load()
        self.ptrs = []

    def put(self, a: np.ndarray) -> int:
        ptr = self.lib.gpudb_host_alloc(max(16, a.nbytes))
        assert ptr
        if a.nbytes:
            np.ctypeslib.as_array((C.c_uint8 * a.nbytes).from_address(ptr))[:] = a.view(np.uint8)
        self.ptrs.append(ptr)
        return ptr

    def columns(self, table: dict, in_place=()) -> list:
        return [(c, self.put(a), a.itemsize, c in in_place) for c, a in table.items()]

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        for p in self.ptrs:
            self.lib.gpudb_host_free(C.c_void_p(p))


@pytest.fixture(scope="module")
def join_data():
    d = W.gen_dim(200_000, seed=5)
    p = W.gen_probe(1_000_003, dim_rows=200_000, seed=5)
    return d, p, O.join_topk(d, p, k=10)


@pytest.mark.parametrize("chunk", [300_001, 1 << 20, 5_000_000])
@pytest.mark.parametrize("in_place", [("p_price", "p_discount"), ()])
def test_streamed_join_topk(ctx, join_data, chunk, in_place):
    d, p, (top, _, distinct) = join_data
    ctx.upload_table("dim", d)
    with Pinned() as pin:
        cols = pin.columns(p, in_place)
        for tune in ("split=0", "split=0;stages=2;warp=0"):
            res, t = ctx.run_streamed("template=join_topk", "probe", cols, len(p["p_fk"]), chunk, tune=tune)
            assert t.device_error == 0
            assert res.rows == top
            assert ctx.get_symbol("jt_groups") == distinct
    # the streamed chunks are not left registered: a resident run needs the table again
    with pytest.raises(GpudbError):
        ctx.run("template=join_topk", "split=0")
    ctx.upload_table("probe", p)
    res, _ = ctx.run("template=join_topk", "split=0")
    assert res.rows == top


def test_streamed_run_refusals(ctx, join_data):
    d, p, _ = join_data
    ctx.upload_table("dim", d)
    with Pinned() as pin:
        cols = pin.columns(p, ("p_price", "p_discount"))
        # the split plan's group phase reads the probe table after the stream
        with pytest.raises(GpudbError, match="outside the streamed phases"):
            ctx.run_streamed("template=join_topk", "probe", cols, len(p["p_fk"]), 1 << 18, tune="split=1")
        # every column the streamed phases read must be supplied
        with pytest.raises(GpudbError, match="not supplied"):
            ctx.run_streamed("template=join_topk", "probe", cols[:3], len(p["p_fk"]), 1 << 18, tune="split=0")
        # no phase scans the named table
        with pytest.raises(GpudbError, match="no phase"):
            ctx.run_streamed("template=join_topk", "fact", cols, len(p["p_fk"]), 1 << 18, tune="split=0")
        # a column read by every row cannot stay on the host
        bad = [(c, ptr, e, c == "p_fk") for c, ptr, e, _ in cols]
        with pytest.raises(GpudbError):
            ctx.run_streamed("template=join_topk", "probe", bad, len(p["p_fk"]), 1 << 18, tune="split=0")
    # the context still answers correctly afterwards
    ctx.upload_table("probe", p)
    res, _ = ctx.run("template=join_topk", "split=0")
    assert res.rows == join_data[2][0]


@pytest.mark.parametrize("n,chunk", [(1_000_003, 262_147), (300_000, 1 << 22), (0, 4096), (5, 2)])
def test_streamed_q1_q6(ctx, n, chunk):
    f = W.gen_fact(n, seed=17)
    q1, q6 = O.q1(f), O.q6(f)
    with Pinned() as pin:
        cols = pin.columns(f)
        for tune in ("", "keyed=5;bs=256;tile=448;stages=2;occ=2;vec=2;l2pf=1", "scan=direct"):
            res, t = ctx.run_streamed("template=q1", "fact", cols, n, chunk, tune=tune)
            assert t.device_error == 0
            assert_q1_equal(res, q1)
        res, _ = ctx.run_streamed("template=q6", "fact", cols, n, chunk)
        assert res.rows == [(q6,)]
