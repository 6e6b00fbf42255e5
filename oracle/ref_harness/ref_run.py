"""Run the reference engine's own generated kernels on the CPU — TEST
INFRASTRUCTURE (oracle pinning).

Loads oracle/_ref/libref_kernels.so (built by build_ref.py from the
reference's code generator) and executes its phases over numpy buffers laid
out per oracle/_ref/manifest.json, exactly as the reference executor binds
them (metal_generic_executor.cpp: allocatePhaseBuffers :74-158 — buffers
from symbolic sizes, zero / 0xFF fill; TableSize as a uint). Decoding of the
outputs follows the reference's result collector
(metal_result_collector.cpp: lo/hi reconstruction :129-132, keyed buckets
with all-zero buckets skipped :204-269, scalar aggregates :157-198).

Inputs take the reference's column types: decimals as float32 in currency
units (price cents/100, discount and tax hundredths/100), the reference's
FP32 fixed-point arithmetic then applies. Threadgroup count is reduced for
CPU speed (integer results do not depend on it).
"""
from __future__ import annotations

import ctypes as C
import json
from pathlib import Path
from typing import Dict

import numpy as np

REF_OUT = Path(__file__).resolve().parent.parent / "_ref"

_ELEM = {"float": np.float32, "int": np.int32, "uint": np.uint32, "char": np.int8, "uchar": np.uint8,
         "long": np.int64, "ulong": np.uint64, "atomic_uint": np.uint32, "atomic_int": np.int32,
         "atomic_float": np.float32}


def available() -> bool:
    return (REF_OUT / "libref_kernels.so").exists() and (REF_OUT / "manifest.json").exists()


class RefKernels:
    def __init__(self):
        self.lib = C.CDLL(str(REF_OUT / "libref_kernels.so"))
        self.manifest = json.loads((REF_OUT / "manifest.json").read_text())

    def run(self, plan: str, columns: Dict[str, np.ndarray], rows: Dict[str, int], symbols: Dict[str, int],
            scalars: Dict[str, int] | None = None, num_tg: int = 8, tg_size: int = 256) -> Dict[str, np.ndarray]:
        """Execute every phase of `plan`; returns the allocated buffers by name."""
        scalars = scalars or {}
        env = dict(symbols)
        for t, n in rows.items():
            env["n_" + t] = n
            env["num" + t] = n
        buffers: Dict[str, np.ndarray] = {}
        for ph in self.manifest[plan]["phases"]:
            args = (C.c_void_p * len(ph["bindings"]))()
            keep = []
            for b in ph["bindings"]:
                kind, name = b["kind"], b["name"]
                if kind == "TableData":
                    arr = np.ascontiguousarray(columns[name])
                elif kind == "TableSize":
                    arr = np.array([rows[b["table"]]], dtype=np.uint32)
                elif kind == "ConstantScalar":
                    arr = np.array([scalars[name]], dtype=_ELEM.get(b["elem"], np.int32))
                elif kind == "DeviceBuffer":
                    if name not in buffers:
                        count = max(1, int(eval(b["size"], {"__builtins__": {}}, env))) if b["size"] else 1
                        dt = _ELEM[b["elem"].replace("const ", "")]
                        buf = np.zeros(count, dtype=dt)
                        if b["zeroInit"] and b["fill"]:
                            buf.view(np.uint8)[:] = b["fill"]
                        buffers[name] = buf
                    arr = buffers[name]
                else:
                    raise ValueError(f"unsupported binding kind {kind}")
                keep.append(arr)
                args[b["index"]] = arr.ctypes.data
            tg = min(tg_size, ph["threadgroupSize"])
            getattr(self.lib, "ref_" + ph["name"])(args, C.c_uint(num_tg), C.c_uint(tg))
        return buffers

    # -- decoding, following the reference's result collector ------------
    def keyed(self, plan: str, buffers) -> list:
        s = self.manifest[plan]["schema"]["keyed"]
        data = buffers[s["buffer"]].view(np.uint32)
        out = []
        for b in range(s["numBuckets"]):
            row = data[b * s["valuesPerBucket"]:(b + 1) * s["valuesPerBucket"]]
            if not row.any():
                continue  # empty bucket
            r = {"bucket": b}
            for sl in s["slots"]:
                if sl["isLongPair"]:
                    v = int(np.int64((int(row[sl["offset"] + 1]) << 32) | int(row[sl["offset"]])))
                else:
                    v = int(row[sl["offset"]])
                r[sl["name"]] = v
            out.append(r)
        return out

    def scalar(self, plan: str, buffers) -> dict:
        out = {}
        for e in self.manifest[plan]["schema"]["scalar"]:
            lo = int(buffers[e["lo"]].view(np.uint32)[0])
            if e["isLongPair"]:
                hi = int(buffers[e["hi"]].view(np.uint32)[0])
                out[e["name"]] = int(np.int64((hi << 32) | lo))
            else:
                out[e["name"]] = float(buffers[e["lo"]].view(np.float32)[0])
        return out


def fact_as_reference(fact: Dict[str, np.ndarray]) -> Dict[str, np.ndarray]:
    """Config-0 columns in the reference's lineitem schema (tpch_schema.h:75-85)."""
    return {"l_shipdate": fact["f_ship_day"].astype(np.int32),
            "l_quantity": fact["f_quantity"].astype(np.float32),
            "l_extendedprice": (fact["f_price"] / 100.0).astype(np.float32),
            "l_discount": (fact["f_discount"] / 100.0).astype(np.float32),
            "l_tax": (fact["f_tax"] / 100.0).astype(np.float32),
            "l_returnflag": fact["f_flag_a"].view(np.int8),
            "l_linestatus": fact["f_flag_b"].view(np.int8)}


def snow_as_reference(snow: Dict[str, Dict[str, np.ndarray]], day_ge: int = 730, day_lt: int = 1095):
    """The multi-join snowflake in the reference's Q5 schema (nation,
    customer, supplier, orders, lineitem; metal_plan_builder.cpp:894-1015).
    The reference's Q5 plan filters o_orderdate on yyyymmdd literals
    [19940101, 19950101); the day numbers are mapped onto that scale by a
    monotone map that sends [day_ge, day_lt) exactly onto it, so the same
    orders qualify. Returns (columns, rows, symbols)."""
    nat, cust, supp, ords, line = (snow[t] for t in ("nation", "cust", "supp", "ord", "line"))
    d = ords["o_day"].astype(np.int64)
    date = np.where(d < day_ge, 19930000 + d - day_ge,
                    np.where(d < day_lt, 19940101 + d - day_ge, 19950101 + d - day_lt))
    cols = {"n_nationkey": nat["n_key"].astype(np.int32), "n_regionkey": nat["n_region"].astype(np.int32),
            "c_custkey": cust["c_key"], "c_nationkey": cust["c_nation"],
            "s_suppkey": supp["s_key"], "s_nationkey": supp["s_nation"],
            "o_orderkey": ords["o_key"], "o_custkey": ords["o_cust"], "o_orderdate": date.astype(np.int32),
            "l_orderkey": line["l_okey"], "l_suppkey": line["l_supp"],
            "l_extendedprice": (line["l_price"] / 100.0).astype(np.float32),
            "l_discount": (line["l_discount"] / 100.0).astype(np.float32)}
    rows = {"nation": 25, "customer": len(cust["c_key"]), "supplier": len(supp["s_key"]),
            "orders": len(ords["o_key"]), "lineitem": len(line["l_okey"])}
    top = lambda *a: int(max(int(x.max(initial=0)) for x in a)) + 1  # noqa: E731
    syms = {"maxCustkey": top(cust["c_key"], ords["o_cust"]), "maxSuppkey": top(supp["s_key"], line["l_supp"]),
            "maxOrderkey": top(ords["o_key"], line["l_okey"])}
    return cols, rows, syms
