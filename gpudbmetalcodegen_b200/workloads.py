"""Seeded synthetic tables for the measured workloads (numpy, via libgpudb's
generators in include/gpudb_datagen.h) and their registration.

Workloads (sizes from the benchmark configurations this backend is measured on):
  scan_filter_groupagg  fact 6,001,215 rows x 38 B
  join_topk             dim 15M rows (key, order_day, segment) + probe 60M rows (fk, ship_day, price, discount)
  skew                  zbuild 2^22 keys + zprobe 120M rows, Zipf(1.1) keys
  mix                   mix table up to 120M rows + mixdim
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


def _alloc(cols, n):
    return {k: np.empty(n, dtype=v) for k, v in cols.items()}


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


def gen_fact(n: int = FACT_ROWS, seed: int = SEED, row0: int = 0, threads: int = 0) -> Dict[str, np.ndarray]:
    t = _alloc(FACT_COLUMNS, n)
    st = _lib.load().gpudb_gen_fact(seed, row0, n, *(_p(t[c]) for c in FACT_COLUMNS), threads)
    assert st == 0
    return t


def gen_dim(n: int = DIM_ROWS, seed: int = SEED, row0: int = 0, count: int = -1,
            threads: int = 0) -> Dict[str, np.ndarray]:
    count = n - row0 if count < 0 else count
    t = _alloc(DIM_COLUMNS, count)
    st = _lib.load().gpudb_gen_dim(seed, n, row0, count, *(_p(t[c]) for c in DIM_COLUMNS), threads)
    assert st == 0
    return t


def gen_probe(n: int = PROBE_ROWS, dim_rows: int = DIM_ROWS, seed: int = SEED, row0: int = 0,
              threads: int = 0) -> Dict[str, np.ndarray]:
    t = _alloc(PROBE_COLUMNS, n)
    st = _lib.load().gpudb_gen_probe(seed, dim_rows, row0, n, *(_p(t[c]) for c in PROBE_COLUMNS), threads)
    assert st == 0
    return t


def gen_zbuild(nkeys: int = ZKEYS, seed: int = SEED, threads: int = 0) -> Dict[str, np.ndarray]:
    t = _alloc(ZBUILD_COLUMNS, nkeys)
    st = _lib.load().gpudb_gen_zbuild(seed, 0, nkeys, _p(t["zb_key"]), _p(t["zb_payload"]), threads)
    assert st == 0
    return t


def gen_zprobe(n: int = ZPROBE_ROWS, nkeys: int = ZKEYS, s: float = ZIPF_S, seed: int = SEED, row0: int = 0,
               threads: int = 0) -> Dict[str, np.ndarray]:
    t = _alloc(ZPROBE_COLUMNS, n)
    st = _lib.load().gpudb_gen_zprobe(seed, nkeys, s, row0, n, _p(t["z_key"]), _p(t["z_value"]), threads)
    assert st == 0
    return t


def gen_mix(n: int, nranks: int = 1 << 22, s: float = ZIPF_S, dim_rows: int = 1_000_000, seed: int = SEED,
            row0: int = 0, threads: int = 0) -> Dict[str, np.ndarray]:
    t = _alloc(MIX_COLUMNS, n)
    st = _lib.load().gpudb_gen_mix(seed, nranks, s, dim_rows, row0, n, *(_p(t[c]) for c in MIX_COLUMNS), threads)
    assert st == 0
    return t


def gen_mixdim(n: int = 1_000_000, seed: int = SEED, threads: int = 0) -> Dict[str, np.ndarray]:
    t = _alloc(MIXDIM_COLUMNS, n)
    st = _lib.load().gpudb_gen_mixdim(seed, 0, n, _p(t["md_key"]), _p(t["md_attr"]), threads)
    assert st == 0
    return t


def table_bytes(t: Dict[str, np.ndarray]) -> int:
    return sum(a.nbytes for a in t.values())
