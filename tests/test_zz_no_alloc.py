"""Allocation-free distinct count, called through the C-ABI.

Some callers of this library cannot allocate device memory on their call
path: a host (a database buffer manager, a JNI/cgo embedding) whose own
allocator owns all device memory. For them gpudb_distinct_count_noalloc keeps its scratch
bitmap in a static device array instead of allocating. This test checks it
against the allocating "distinct" pipeline (gpudb_query_run) on the same
device columns, on two calls in a row, and checks that a cardinality above
the static scratch's limit is rejected. It lives in its own file, collected
last, and passes alone in a fresh process as well as after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_distinct_matches_the_allocating_pipeline():
    torch = pytest.importorskip("torch")
    from gpudbmetalcodegen_b200 import Context, _lib
    from gpudbmetalcodegen_b200 import workloads as W

    lib = _lib.load()
    n = 300_000
    mix = W.gen_mix(n, nranks=1 << 20, dim_rows=1000, seed=21)
    with Context(0) as ctx:
        cols = {c: torch.from_numpy(a).cuda() for c, a in mix.items()}
        torch.cuda.synchronize()
        for c, t in cols.items():
            ctx.register_tensor("mix", c, t)
        out = torch.zeros(1, dtype=torch.int64, device="cuda")
        for key, thr, card in (("m_rank_u", 5000, 1000), ("m_rank_z", 9000, 1 << 22), ("m_rank_u", 1, 77)):
            res, _ = ctx.run(f"template=distinct;key={key};thr={thr};card={card}")
            expect = res.rows[0][0]
            sel = mix["m_filter"] < thr
            assert expect == np.unique(mix[key][sel].astype(np.int64) % card).shape[0]
            for _ in range(2):
                out.fill_(-1)
                torch.cuda.synchronize()
                st = lib.gpudb_distinct_count_noalloc(C.c_void_p(cols[key].data_ptr()),
                                                      C.c_void_p(cols["m_filter"].data_ptr()), n, thr, card,
                                                      C.c_void_p(out.data_ptr()), C.c_void_p(ctx.stream_ptr))
                assert st == 0, _lib.last_error(None)
                ctx.synchronize()
                assert int(out.item()) == expect

        # no rows: the count is 0 (the scratch still holds the last call's bits)
        out.fill_(-1)
        torch.cuda.synchronize()
        st = lib.gpudb_distinct_count_noalloc(C.c_void_p(cols["m_rank_u"].data_ptr()),
                                              C.c_void_p(cols["m_filter"].data_ptr()), 0, 5000, 1000,
                                              C.c_void_p(out.data_ptr()), C.c_void_p(ctx.stream_ptr))
        assert st == 0, _lib.last_error(None)
        ctx.synchronize()
        assert int(out.item()) == 0

        st = lib.gpudb_distinct_count_noalloc(C.c_void_p(cols["m_rank_u"].data_ptr()),
                                              C.c_void_p(cols["m_filter"].data_ptr()), n, 5000, (1 << 22) + 1,
                                              C.c_void_p(out.data_ptr()), C.c_void_p(ctx.stream_ptr))
        assert st == -1
        assert "2^22" in _lib.last_error(None)
