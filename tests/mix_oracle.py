"""Oracle answers of mixed-workload queries — TEST INFRASTRUCTURE.

A query's slice is taken from the table's host copy when the MixTables
keeps one, else regenerated on the host from the same seeds (every value
is a pure function of seed, column and row), then the oracle computes the
answer in the form BatchRunner returns it.
"""
from gpudbmetalcodegen_b200 import batch as B
from gpudbmetalcodegen_b200 import workloads as W
from oracle import oracle_py as O

_dims = {}


def slice_of(tables, q):
    if tables.host:
        return tables.slice_host(q)
    return W.gen_mix(q.rows, nranks=tables.nranks, s=tables.zipf_s[q.table], dim_rows=tables.dim_rows,
                     seed=tables.table_seed(q.table), row0=q.row0)


def dim_of(tables):
    if tables.dim_host is not None:
        return tables.dim_host
    key = (tables.seed, tables.dim_rows)
    if key not in _dims:
        _dims[key] = W.gen_mixdim(tables.dim_rows, seed=tables.seed)
    return _dims[key]


def oracle_result(tables, q):
    m = slice_of(tables, q)
    if q.tmpl == "agg":
        c, s = O.mix_agg(m, q.thr)
        return ("scalar", c, s)
    if q.tmpl == "join":
        c, s = O.mix_join(dim_of(tables), m, q.attr_lt, q.thr)
        return ("scalar", c, s)
    k, c, s = O.mix_groupby(m, q.key, q.thr, q.card)
    if q.tmpl == "groupby":
        return B.canonical_groups(k, c, s)
    return ("topk", tuple(O.topk(k, s, q.k)))
