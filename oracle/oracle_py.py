"""ctypes wrapper of the CPU oracle (liboracle.so) — TEST INFRASTRUCTURE.

Imported only by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg, as the checker / the timed CPU restatement; never by the
product package.
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, List, Tuple

import numpy as np

from . import build_oracle


class I128(C.Structure):
    _fields_ = [("lo", C.c_uint64), ("hi", C.c_int64)]

    def value(self) -> int:
        return (self.hi << 64) | self.lo


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        path = build_oracle.build()
        _lib = C.CDLL(str(path))
        P = C.c_void_p
        sig = {
            "oracle_q1": (C.c_int, [C.c_uint64] + [P] * 7 + [C.c_int32, P, C.c_int]),
            "oracle_q6": (C.c_int, [C.c_uint64] + [P] * 4 + [C.c_int32, C.c_int32, C.c_int64, C.c_int64, C.c_int64,
                                                            P, C.c_int]),
            "oracle_join_topk": (C.c_int, [C.c_uint64, P, P, P, C.c_uint64, P, P, P, P, C.c_int32, C.c_int32,
                                           C.c_int32, C.c_int, P, P, P, P, C.c_int]),
            "oracle_groupby": (C.c_int64, [C.c_uint64, P, P, C.c_uint64, P, P, P, C.c_int]),
            "oracle_hashjoin": (C.c_int64, [C.c_uint64, P, P, C.c_uint64, P, C.c_uint64, P, P, P, C.c_int]),
            "oracle_mix_agg": (C.c_int, [C.c_uint64, P, P, C.c_int32, P, P, C.c_int]),
            "oracle_mix_groupby": (C.c_int64, [C.c_uint64, P, P, P, C.c_int32, C.c_int64, C.c_uint64, P, P, P,
                                               C.c_int]),
            "oracle_mix_join": (C.c_int, [C.c_uint64, P, P, C.c_int32, C.c_uint64, P, P, P, C.c_int32, P, P,
                                          C.c_int]),
            "oracle_topk": (C.c_int, [C.c_uint64, P, P, C.c_int, P, P]),
            "oracle_max_i32": (C.c_int64, [C.c_uint64, P, C.c_int]),
            "oracle_anti_join": (C.c_int, [C.c_uint64, P, P, P, C.c_uint64, P, P, P, P, C.c_int32, C.c_int32,
                                           C.c_int32, C.c_int, P, P, C.c_int]),
            "oracle_histogram": (C.c_int, [C.c_uint64, P, C.c_uint64, P, P, C.c_int32, C.c_int, P, C.c_int]),
        }
        for name, (res, args) in sig.items():
            f = getattr(_lib, name)
            f.restype = res
            f.argtypes = args
    return _lib


def _p(a):
    return a.ctypes.data


Q1_AGGS = ["sum_qty", "sum_base_price", "sum_disc_price", "sum_charge", "sum_disc", "count_order"]
FLAG_A = "ANR"
FLAG_B = "FO"


def q1(fact: Dict[str, np.ndarray], ship_le: int = 2436, threads: int = 0) -> List[dict]:
    """Rows in bucket order, empty groups omitted, FP64 averages derived once."""
    out = (I128 * 36)()
    n = fact["f_ship_day"].shape[0]
    lib().oracle_q1(n, _p(fact["f_ship_day"]), _p(fact["f_quantity"]), _p(fact["f_price"]), _p(fact["f_discount"]),
                    _p(fact["f_tax"]), _p(fact["f_flag_a"]), _p(fact["f_flag_b"]), ship_le, out, threads)
    rows = []
    for b in range(6):
        v = [out[b * 6 + j].value() for j in range(6)]
        if not any(v):
            continue
        r = {"flag_a": FLAG_A[(b // 2) % 3], "flag_b": FLAG_B[b % 2]}
        r.update(dict(zip(Q1_AGGS, v)))
        c = r["count_order"]
        r["avg_qty"] = float(r["sum_qty"]) / float(c)
        r["avg_price"] = float(r["sum_base_price"]) / float(c)
        r["avg_disc"] = float(r["sum_disc"]) / float(c)
        rows.append(r)
    return rows


def q6(fact, ship_ge=365, ship_lt=730, disc_lo=5, disc_hi=7, qty_lt=24, threads: int = 0) -> int:
    out = I128()
    n = fact["f_ship_day"].shape[0]
    lib().oracle_q6(n, _p(fact["f_ship_day"]), _p(fact["f_quantity"]), _p(fact["f_price"]), _p(fact["f_discount"]),
                    ship_ge, ship_lt, disc_lo, disc_hi, qty_lt, C.byref(out), threads)
    return out.value()


def join_topk(dim, probe, seg=1, od_lt=1170, ship_gt=1170, k=10, threads: int = 0) -> Tuple[List[tuple], int, int]:
    keys = np.zeros(k, np.int64)
    vals = np.zeros(k, np.int64)
    groups = C.c_uint64()
    distinct = C.c_uint64()
    cnt = lib().oracle_join_topk(dim["b_key"].shape[0], _p(dim["b_key"]), _p(dim["b_order_day"]),
                                 _p(dim["b_segment"]), probe["p_fk"].shape[0], _p(probe["p_fk"]),
                                 _p(probe["p_ship_day"]), _p(probe["p_price"]), _p(probe["p_discount"]), seg, od_lt,
                                 ship_gt, k, _p(keys), _p(vals), C.byref(groups), C.byref(distinct), threads)
    assert cnt >= 0
    return [(int(keys[i]), int(vals[i])) for i in range(cnt)], groups.value, distinct.value


def join_rows(dim, probe, seg=1, od_lt=1170, ship_gt=1170) -> List[tuple]:
    """The rows of the Q3-shape semi-join, materialised instead of
    aggregated: (probe row, key, price * (100 - discount)) for every probe
    row with ship_day > ship_gt whose key is a build key with segment == seg
    and order_day < od_lt (reference: MetalMaterialize,
    metal_operators.cpp:618-643, over the join of
    metal_plan_builder.cpp:1170-1239). Sorted by row: the engine's output
    order is unspecified, as the reference's atomic positions are. numpy,
    exact int64."""
    keep = (dim["b_segment"] == seg) & (dim["b_order_day"] < od_lt)
    top = int(max(int(dim["b_key"].max(initial=0)), int(probe["p_fk"].max(initial=0)))) + 1
    qual = np.zeros(top + 1, dtype=bool)
    qual[dim["b_key"][keep]] = True
    fk = probe["p_fk"]
    ok = (probe["p_ship_day"] > ship_gt) & (fk >= 0) & qual[np.clip(fk, 0, top)]
    rows = np.nonzero(ok)[0]
    rev = probe["p_price"][rows] * (100 - probe["p_discount"][rows])
    return [(int(r), int(k), int(v)) for r, k, v in zip(rows, fk[rows], rev)]


def groupby(key: np.ndarray, value: np.ndarray, cap: int, threads: int = 0):
    ok, oc, os_ = (np.zeros(cap, np.int64) for _ in range(3))
    g = lib().oracle_groupby(key.shape[0], _p(key), _p(value), cap, _p(ok), _p(oc), _p(os_), threads)
    assert g >= 0, "oracle group-by capacity exceeded"
    return ok[:g], oc[:g], os_[:g]


def hashjoin(zbuild, probe_key: np.ndarray, cap: int, threads: int = 0):
    ok, oc, os_ = (np.zeros(cap, np.int64) for _ in range(3))
    g = lib().oracle_hashjoin(zbuild["zb_key"].shape[0], _p(zbuild["zb_key"]), _p(zbuild["zb_payload"]),
                              probe_key.shape[0], _p(probe_key), cap, _p(ok), _p(oc), _p(os_), threads)
    assert g >= 0
    return ok[:g], oc[:g], os_[:g]


def mix_agg(mix, thr: int, threads: int = 0) -> Tuple[int, int]:
    c = C.c_int64()
    s = I128()
    lib().oracle_mix_agg(mix["m_filter"].shape[0], _p(mix["m_filter"]), _p(mix["m_value"]), thr, C.byref(c),
                         C.byref(s), threads)
    return c.value, s.value()


def mix_groupby(mix, key_col: str, thr: int, card: int, threads: int = 0):
    n = mix["m_filter"].shape[0]
    cap = max(1, min(n, card))
    ok, oc, os_ = (np.zeros(cap, np.int64) for _ in range(3))
    g = lib().oracle_mix_groupby(n, _p(mix[key_col]), _p(mix["m_filter"]), _p(mix["m_value"]), thr, card, cap,
                                 _p(ok), _p(oc), _p(os_), threads)
    assert g >= 0
    return ok[:g], oc[:g], os_[:g]


def mix_join(mixdim, mix, attr_lt: int, thr: int, threads: int = 0) -> Tuple[int, int]:
    c = C.c_int64()
    s = I128()
    lib().oracle_mix_join(mixdim["md_key"].shape[0], _p(mixdim["md_key"]), _p(mixdim["md_attr"]), attr_lt,
                          mix["m_fk"].shape[0], _p(mix["m_fk"]), _p(mix["m_filter"]), _p(mix["m_value"]), thr,
                          C.byref(c), C.byref(s), threads)
    return c.value, s.value()


def topk(keys: np.ndarray, vals: np.ndarray, k: int) -> List[tuple]:
    keys = np.ascontiguousarray(keys, dtype=np.int64)
    vals = np.ascontiguousarray(vals, dtype=np.int64)
    ok = np.zeros(k, np.int64)
    ov = np.zeros(k, np.int64)
    n = lib().oracle_topk(keys.shape[0], _p(keys), _p(vals), k, _p(ok), _p(ov))
    return [(int(ok[i]), int(ov[i])) for i in range(n)]


def max_i32(v: np.ndarray, threads: int = 0) -> int:
    return int(lib().oracle_max_i32(v.shape[0], _p(v), threads))


def join_direct(dim, probe, seg=1, od_lt=1170, ship_gt=1170, k=10, threads: int = 0) -> List[tuple]:
    """The Q3 operator chain's answer (metal_plan_builder.cpp:1170-1239 with
    the host top-k of codegen_main.cpp:1211-1248, ties by key): the join's
    top k (key, revenue) with the matched build row's order_day and
    segment, read from the build table as the reference reads its maps."""
    top, _, _ = join_topk(dim, probe, seg, od_lt, ship_gt, k, threads)
    if not top:
        return []
    keys = dim["b_key"]
    order = np.argsort(keys, kind="stable")
    pos = order[np.searchsorted(keys[order], [t[0] for t in top])]
    return [(key, rev, int(dim["b_order_day"][p]), int(dim["b_segment"][p])) for (key, rev), p in zip(top, pos)]


def anti_join(dim, probe, seg=1, od_lt=1170, ship_gt=1170, nbins=11, threads: int = 0) -> List[tuple]:
    """Rows (discount, count, sum_price) of non-empty bins, in bin order."""
    cnt = np.zeros(nbins, np.int64)
    sums = (I128 * nbins)()
    st = lib().oracle_anti_join(dim["b_key"].shape[0], _p(dim["b_key"]), _p(dim["b_order_day"]),
                                _p(dim["b_segment"]), probe["p_fk"].shape[0], _p(probe["p_fk"]),
                                _p(probe["p_ship_day"]), _p(probe["p_price"]), _p(probe["p_discount"]), seg, od_lt,
                                ship_gt, nbins, _p(cnt), sums, threads)
    if st != 0:
        raise ValueError("anti_join: a bin lies outside [0, nbins)")
    return [(b, int(cnt[b]), sums[b].value()) for b in range(nbins) if cnt[b] or sums[b].value()]


def histogram(dim, probe, ship_gt=1170, nbins=256, threads: int = 0) -> List[tuple]:
    """Rows (rows_per_key, keys) of non-empty bins, in bin order."""
    hist = np.zeros(nbins, np.int64)
    st = lib().oracle_histogram(dim["b_key"].shape[0], _p(dim["b_key"]), probe["p_fk"].shape[0], _p(probe["p_fk"]),
                                _p(probe["p_ship_day"]), ship_gt, nbins, _p(hist), threads)
    if st != 0:
        raise ValueError("histogram: a probe key beyond the build keys, or a count beyond the bins")
    return [(c, int(hist[c])) for c in range(nbins) if hist[c]]


def multi_join(snow, region=2, day_ge=730, day_lt=1095) -> List[tuple]:
    """The reference's Q5 plan shape (metal_plan_builder.cpp:894-1015) over
    the snowflake: nations of `region`; customers and suppliers of those
    nations; orders with day_ge <= day < day_lt and such a customer; lines
    of those orders whose supplier's nation equals the customer's nation;
    per nation the exact sum of price * (100 - discount). Rows (nation,
    revenue) of non-zero nations in nation order. numpy, exact int64."""
    nat = snow["nation"]
    in_region = np.zeros(25, dtype=bool)
    in_region[nat["n_key"][nat["n_region"] == region]] = True
    cust, supp, ords, line = snow["cust"], snow["supp"], snow["ord"], snow["line"]
    cn = np.full(int(cust["c_key"].max(initial=0)) + 1, -1, np.int64)
    keep = in_region[cust["c_nation"]]
    cn[cust["c_key"][keep]] = cust["c_nation"][keep]
    sn = np.full(int(supp["s_key"].max(initial=0)) + 1, -1, np.int64)
    keep = in_region[supp["s_nation"]]
    sn[supp["s_key"][keep]] = supp["s_nation"][keep]
    on = np.full(int(ords["o_key"].max(initial=0)) + 1, -1, np.int64)
    dk = (ords["o_day"] >= day_ge) & (ords["o_day"] < day_lt)
    c_of = cn[ords["o_cust"][dk]]
    on[ords["o_key"][dk][c_of >= 0]] = c_of[c_of >= 0]
    lc = on[line["l_okey"]]
    ls = sn[line["l_supp"]]
    ok = (lc >= 0) & (lc == ls)
    rev = line["l_price"][ok] * (100 - line["l_discount"][ok])
    sums = np.zeros(25, np.int64)
    np.add.at(sums, lc[ok], rev)
    return [(n, int(sums[n])) for n in range(25) if sums[n]]
