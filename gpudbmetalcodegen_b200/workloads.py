"""Seeded synthetic tables for the measured workloads (numpy, via the
generators of libgpudb_datagen.so, include/gpudb_datagen.h) and their
registration.

Workloads (sizes from the benchmark configurations this backend is measured on):
  scan_filter_groupagg  fact 6,001,215 rows x 38 B
  join_topk             dim 15M rows (key, order_day, segment) + probe 60M rows (fk, ship_day, price, discount)
  skew                  zbuild 2^22 keys + zprobe 120M rows, Zipf(1.1) keys
  mix                   mix table up to 120M rows + mixdim
  multi_join            the snowflake nation (25) / cust / supp / ord / line (the Q5 shape)
"""
from __future__ import annotations

import ctypes as C
from typing import Dict

import numpy as np

from . import _lib

SEED = 20240501
FACT_ROWS = 6_001_215
DIM_ROWS = 15_000_000
PROBE_ROWS = 60_000_000
ZKEYS = 1 << 22
ZPROBE_ROWS = 120_000_000
ZIPF_S = 1.1

FACT_COLUMNS = {"f_ship_day": np.int32, "f_quantity": np.int64, "f_price": np.int64, "f_discount": np.int64,
                "f_tax": np.int64, "f_flag_a": np.uint8, "f_flag_b": np.uint8}
DIM_COLUMNS = {"b_key": np.int32, "b_order_day": np.int32, "b_segment": np.uint8}
PROBE_COLUMNS = {"p_fk": np.int32, "p_ship_day": np.int32, "p_price": np.int64, "p_discount": np.int64}
ZBUILD_COLUMNS = {"zb_key": np.int64, "zb_payload": np.int32}
ZPROBE_COLUMNS = {"z_key": np.int64, "z_value": np.int64}
MIX_COLUMNS = {"m_rank_u": np.int32, "m_rank_z": np.int32, "m_filter": np.int32, "m_value": np.int64,
               "m_fk": np.int32}
MIXDIM_COLUMNS = {"md_key": np.int32, "md_attr": np.int32}
SNOW_CUST_ROWS, SNOW_SUPP_ROWS, SNOW_ORDER_ROWS, SNOW_LINE_ROWS = 1_500_000, 100_000, 15_000_000, 60_000_000
LINE_COLUMNS = {"l_okey": np.int32, "l_supp": np.int32, "l_price": np.int64, "l_discount": np.int64}


def _alloc(cols, n):
    return {k: np.empty(n, dtype=v) for k, v in cols.items()}


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


def gen_fact(n: int = FACT_ROWS, seed: int = SEED, row0: int = 0, threads: int = 0) -> Dict[str, np.ndarray]:
    t = _alloc(FACT_COLUMNS, n)
    st = _lib.load_datagen().gpudb_gen_fact(seed, row0, n, *(_p(t[c]) for c in FACT_COLUMNS), threads)
    assert st == 0
    return t


def gen_dim(n: int = DIM_ROWS, seed: int = SEED, row0: int = 0, count: int = -1,
            threads: int = 0) -> Dict[str, np.ndarray]:
    count = n - row0 if count < 0 else count
    t = _alloc(DIM_COLUMNS, count)
    st = _lib.load_datagen().gpudb_gen_dim(seed, n, row0, count, *(_p(t[c]) for c in DIM_COLUMNS), threads)
    assert st == 0
    return t


def gen_probe(n: int = PROBE_ROWS, dim_rows: int = DIM_ROWS, seed: int = SEED, row0: int = 0,
              threads: int = 0) -> Dict[str, np.ndarray]:
    t = _alloc(PROBE_COLUMNS, n)
    st = _lib.load_datagen().gpudb_gen_probe(seed, dim_rows, row0, n, *(_p(t[c]) for c in PROBE_COLUMNS), threads)
    assert st == 0
    return t


def gen_zbuild(nkeys: int = ZKEYS, seed: int = SEED, threads: int = 0) -> Dict[str, np.ndarray]:
    t = _alloc(ZBUILD_COLUMNS, nkeys)
    st = _lib.load_datagen().gpudb_gen_zbuild(seed, 0, nkeys, _p(t["zb_key"]), _p(t["zb_payload"]), threads)
    assert st == 0
    return t


def gen_zprobe(n: int = ZPROBE_ROWS, nkeys: int = ZKEYS, s: float = ZIPF_S, seed: int = SEED, row0: int = 0,
               threads: int = 0) -> Dict[str, np.ndarray]:
    t = _alloc(ZPROBE_COLUMNS, n)
    st = _lib.load_datagen().gpudb_gen_zprobe(seed, nkeys, s, row0, n, _p(t["z_key"]), _p(t["z_value"]), threads)
    assert st == 0
    return t


def gen_mix(n: int, nranks: int = 1 << 22, s: float = ZIPF_S, dim_rows: int = 1_000_000, seed: int = SEED,
            row0: int = 0, threads: int = 0) -> Dict[str, np.ndarray]:
    t = _alloc(MIX_COLUMNS, n)
    st = _lib.load_datagen().gpudb_gen_mix(seed, nranks, s, dim_rows, row0, n, *(_p(t[c]) for c in MIX_COLUMNS), threads)
    assert st == 0
    return t


def gen_mixdim(n: int = 1_000_000, seed: int = SEED, threads: int = 0) -> Dict[str, np.ndarray]:
    t = _alloc(MIXDIM_COLUMNS, n)
    st = _lib.load_datagen().gpudb_gen_mixdim(seed, 0, n, _p(t["md_key"]), _p(t["md_attr"]), threads)
    assert st == 0
    return t


def table_bytes(t: Dict[str, np.ndarray]) -> int:
    return sum(a.nbytes for a in t.values())


# ---------------------------------------------------------------------------
# mixed-query workload: 256 queries over slices of resident mix tables
# ---------------------------------------------------------------------------
MIX_TABLE_ROWS = 120_000_000
MIX_ZIPF_S = (0.8, 0.95, 1.1, 1.3)   # one resident mix table per exponent
MIX_NRANKS = 1 << 22
MIX_DIM_ROWS = 1_000_000
MIX_QUERIES = 256


def gen_mixed_queries(n: int = MIX_QUERIES, seed: int = SEED, table_rows: int = MIX_TABLE_ROWS,
                      n_tables: int = len(MIX_ZIPF_S), min_rows: int = 1_000_000, max_rows: int = 120_000_000,
                      min_card: int = 4, max_card: int = 1 << 22, k: int = 10, templates=None):
    """Seeded mixed queries: template uniform over agg / join / groupby / topk
    (or over `templates`); slice rows log-uniform in [min_rows, max_rows]
    (capped by the table) at a uniform offset of a uniformly chosen table;
    group key uniform (m_rank_u) or Zipf (m_rank_z, the table's exponent)
    with equal odds; cardinality log-uniform in [min_card, max_card]; filter
    selectivity uniform in 1%..99% (m_filter is uniform on 0..9999, so the
    threshold is 100 x the percentage); join keeps md_attr < U[1, 999]."""
    from .batch import MixQuery, TEMPLATES

    templates = tuple(templates or TEMPLATES)
    rng = np.random.default_rng(seed)
    hi = min(max_rows, table_rows)
    lo = min(min_rows, hi)
    out = []
    for _ in range(n):
        tmpl = templates[int(rng.integers(len(templates)))]
        rows = int(round(float(np.exp(rng.uniform(np.log(lo), np.log(hi))))))
        rows = max(1, min(rows, table_rows))
        row0 = int(rng.integers(0, table_rows - rows + 1))
        table = int(rng.integers(n_tables))
        key = "m_rank_z" if rng.random() < 0.5 else "m_rank_u"
        card = int(round(float(np.exp(rng.uniform(np.log(min_card), np.log(max_card))))))
        thr = int(round(rng.uniform(0.01, 0.99) * 10000))
        attr_lt = int(rng.integers(1, 1000))
        out.append(MixQuery(tmpl=tmpl, table=table, row0=row0, rows=rows, thr=thr, key=key, card=card, k=k,
                            attr_lt=attr_lt))
    return out


def gen_snowflake(ncust: int = SNOW_CUST_ROWS, nsupp: int = SNOW_SUPP_ROWS, norders: int = SNOW_ORDER_ROWS,
                  nlines: int = SNOW_LINE_ROWS, seed: int = SEED, threads: int = 0) -> Dict[str, Dict[str, np.ndarray]]:
    """The multi-join snowflake: nation (key 0..24, region key % 5), cust,
    supp, ord and line tables (include/gpudb_datagen.h)."""
    lib = _lib.load_datagen()
    nation = {"n_key": np.arange(25, dtype=np.int32), "n_region": (np.arange(25) % 5).astype(np.int32)}
    cust = {"c_key": np.empty(ncust, np.int32), "c_nation": np.empty(ncust, np.int32)}
    supp = {"s_key": np.empty(nsupp, np.int32), "s_nation": np.empty(nsupp, np.int32)}
    ords = {"o_key": np.empty(norders, np.int32), "o_cust": np.empty(norders, np.int32),
            "o_day": np.empty(norders, np.int32)}
    line = _alloc(LINE_COLUMNS, nlines)
    assert lib.gpudb_gen_snow_cust(seed, 0, ncust, _p(cust["c_key"]), _p(cust["c_nation"]), threads) == 0
    assert lib.gpudb_gen_snow_supp(seed, 0, nsupp, _p(supp["s_key"]), _p(supp["s_nation"]), threads) == 0
    assert lib.gpudb_gen_snow_orders(seed, ncust, 0, norders, _p(ords["o_key"]), _p(ords["o_cust"]),
                                     _p(ords["o_day"]), threads) == 0
    assert lib.gpudb_gen_snow_lines(seed, norders, nsupp, 0, nlines, *(_p(line[c]) for c in LINE_COLUMNS),
                                    threads) == 0
    return {"nation": nation, "cust": cust, "supp": supp, "ord": ords, "line": line}
