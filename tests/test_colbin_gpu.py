""".colbin v2 ingest into HBM on the GPU: the fact table written the way
the reference stores lineitem (quantity INT, price / discount / tax FLOAT,
flags CHAR1, ship date DATE as YYYYMMDD), loaded with the transforms that
give the engine's exact column types, answers Q1 and Q6 exactly as the
same table uploaded directly."""
import numpy as np
import pytest

from colbin_writer import fact_as_lineitem, write_colbin
from gpudbmetalcodegen_b200 import _lib
from gpudbmetalcodegen_b200 import workloads as W
from gpudbmetalcodegen_b200._lib import GpudbError
from oracle import oracle_py as O

pytestmark = pytest.mark.gpu

SPECS = [(4, "f_quantity", _lib.COLBIN_WIDEN, 0), (5, "f_price", _lib.COLBIN_DECIMAL, 100),
         (6, "f_discount", _lib.COLBIN_DECIMAL, 100), (7, "f_tax", _lib.COLBIN_DECIMAL, 100),
         (8, "f_flag_a", _lib.COLBIN_AS_IS, 0), (9, "f_flag_b", _lib.COLBIN_AS_IS, 0),
         (10, "f_ship_day", _lib.COLBIN_DAYS, 0)]


@pytest.mark.parametrize("rows", [0, 1, 4097, 300_000])
def test_colbin_fact_answers_q1_and_q6(ctx, tmp_path, rows):
    fact = W.gen_fact(rows, seed=17)
    p = tmp_path / "lineitem.colbin"
    write_colbin(p, fact_as_lineitem(fact), rows)
    ctx.load_colbin(str(p), "fact", SPECS)
    assert ctx.largest_table_rows() >= rows
    res, t = ctx.run("template=q6")
    assert t.device_error == 0 and res.rows == [(O.q6(fact),)]
    res, _ = ctx.run("template=q1")
    exp = O.q1(fact)
    got = res.as_dicts()
    assert len(got) == len(exp)
    assert all(g[k] == e[k] for g, e in zip(got, exp) for k in O.Q1_AGGS)


def test_colbin_load_rejects_mismatched_columns(ctx, tmp_path):
    fact = W.gen_fact(100, seed=3)
    p = tmp_path / "l.colbin"
    write_colbin(p, fact_as_lineitem(fact), 100)
    with pytest.raises(GpudbError) as e:   # a float column cannot land as is in an int64 column
        ctx.load_colbin(str(p), "fact", [(5, "f_price", _lib.COLBIN_AS_IS, 0)])
    assert "as is" in e.value.message
    with pytest.raises(GpudbError) as e:   # no such source field
        ctx.load_colbin(str(p), "fact", [(42, "f_price", _lib.COLBIN_DECIMAL, 100)])
    assert "no column with source index 42" in e.value.message
