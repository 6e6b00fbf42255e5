"""Batched mixed queries, the learned sizer and the plain per-query path.

Python face of include/gpudb_batch.h. The reference runs one query per
invocation and sizes every table by an exact max-key pass
(codegen/execution/max_key_symbols.cpp:188-235); here many queries of the
four mixed templates run as one set of persistent work-queue kernels, and
their hash tables are sized by an MLP trained on the engine's own logged
executions, with the exact per-query path as fallback when a table
overflows. Every path returns the same canonical results:

    agg / join : ("scalar", count, sum)
    groupby    : ("groups", keys, counts, sums)  numpy int64, sorted by key
    topk       : ("topk", ((key, sum), ...))     best first

The batched path hands group-by results over unsorted, as
("groups_raw", rows[n, 3]) or ("groups_cols", keys, counts, sums) in table
order (a GROUP BY has no row order); `canonical` sorts them when a
comparison needs it.
"""
from __future__ import annotations

import ctypes as C
import math
import threading
import time
import weakref
from dataclasses import dataclass, field, replace
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _lib
from ._lib import check

TEMPLATES = ("agg", "join", "groupby", "topk")
AGG_AUTO, AGG_SHARED, AGG_GLOBAL_WARP, AGG_GLOBAL, AGG_SHARED_DIRECT = 0, 1, 2, 3, 4
DIRECT_MAX_CARD = 1024       # the direct shared table holds keys of (-card, card) in 2048 slots
DIRECT_SKEW_SHARE = 0.01     # top sample-key share above which a small domain counts as skewed
SHARED_MAX_GROUPS = 1024     # groups that fit the per-CTA shared table at load <= 1/2
TPL = {name: i for i, name in enumerate(TEMPLATES)}
DEVERR_HASH_OVERFLOW = 0x1
SIZER_FEATURES = 16
SIZER_OUTPUTS = 2
CARD_SCALE = 24.0  # sizer output 0 = log2(groups + 1) / CARD_SCALE


class BatchQueryStruct(C.Structure):
    """gpudb_batch_query (include/gpudb_batch.h)."""
    _fields_ = [("tmpl", C.c_int), ("thr", C.c_int32), ("card", C.c_int64), ("k", C.c_int32),
                ("attr_lt", C.c_int32), ("rows", C.c_uint64), ("key", C.c_void_p), ("filter", C.c_void_p),
                ("value", C.c_void_p), ("fk", C.c_void_p), ("dim_key", C.c_void_p), ("dim_attr", C.c_void_p),
                ("dim_rows", C.c_uint64), ("dim_max_key", C.c_int64), ("groups", C.c_uint64),
                ("key_min", C.c_int64), ("key_max", C.c_int64), ("filter_min", C.c_int32),
                ("filter_max", C.c_int32), ("agg_mode", C.c_int32)]


QUERY_DTYPE = np.dtype(BatchQueryStruct)  # the same layout as a numpy record


@dataclass(frozen=True)
class MixQuery:
    """One query of the mixed workload over a slice of a resident mix table."""
    tmpl: str                # agg | join | groupby | topk
    table: int               # index of the resident mix table
    row0: int
    rows: int
    thr: int                 # m_filter < thr
    key: str = "m_rank_u"    # group key column: m_rank_u (uniform) or m_rank_z (Zipf)
    card: int = 1            # group key = key % card
    k: int = 10              # top-k
    attr_lt: int = 500       # join: mixdim rows with md_attr < attr_lt

    @property
    def grouped(self) -> bool:
        return self.tmpl in ("groupby", "topk")


# ---------------------------------------------------------------------------
# canonical results
# ---------------------------------------------------------------------------
def canonical_groups(keys, counts, sums):
    keys = np.asarray(keys, dtype=np.int64)
    order = np.argsort(keys, kind="stable")
    return ("groups", keys[order], np.asarray(counts, dtype=np.int64)[order],
            np.asarray(sums, dtype=np.int64)[order])


def canonical(r):
    if r[0] == "groups_raw":
        blk = r[1]
        return canonical_groups(blk[:, 0], blk[:, 1], blk[:, 2])
    if r[0] == "groups_cols":  # (keys, counts, sums) in table order
        return canonical_groups(r[1], r[2], r[3])
    return r


def same_result(a, b) -> bool:
    a, b = canonical(a), canonical(b)
    if a[0] != b[0]:
        return False
    if a[0] == "groups":
        return all(np.array_equal(x, y) for x, y in zip(a[1:], b[1:]))
    return tuple(a[1:]) == tuple(b[1:])


def _mix64(x: np.ndarray) -> np.ndarray:
    x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return x ^ (x >> np.uint64(31))


def result_fingerprint(r) -> tuple:
    """An order-independent 64-bit fingerprint of a result (a multiset hash
    of its group rows, vectorised; exact tuples for scalar / top-k), so
    large answers can be checked without keeping or sorting them."""
    if r[0] == "scalar":
        return r
    if r[0] == "topk":
        return r
    if r[0] == "groups_raw":
        k, c, sm = r[1][:, 0], r[1][:, 1], r[1][:, 2]
    else:
        k, c, sm = r[1], r[2], r[3]
    with np.errstate(over="ignore"):
        k = np.asarray(k).astype(np.uint64)
        c = np.asarray(c).astype(np.uint64)
        sm = np.asarray(sm).astype(np.uint64)
        h = _mix64(k * np.uint64(0x9E3779B97F4A7C15) ^ _mix64(c + np.uint64(1)) ^ _mix64(sm ^ np.uint64(0x5851F42D)))
        return ("groups", int(k.size), int(h.sum(dtype=np.uint64)), int(np.bitwise_xor.reduce(h) if h.size else 0))


def describe_difference(a, b) -> str:
    a, b = canonical(a), canonical(b)
    if a[0] != b[0]:
        return f"kind {a[0]} vs {b[0]}"
    if a[0] == "groups":
        if a[1].shape != b[1].shape:
            return f"{a[1].shape[0]} vs {b[1].shape[0]} groups"
        for name, x, y in zip(("keys", "counts", "sums"), a[1:], b[1:]):
            bad = np.nonzero(x != y)[0]
            if bad.size:
                return f"{name} differ at {bad.size} rows, first row {bad[0]}: {x[bad[0]]} vs {y[bad[0]]}"
        return "equal"
    return f"{a[1:]} vs {b[1:]}"


# ---------------------------------------------------------------------------
# resident tables
# ---------------------------------------------------------------------------
def column_minmax(col, stream=None) -> Tuple[int, int]:
    """(min, max) of a resident int32 / int64 device column, by the
    library's own zone-map kernel (gpudb_column_minmax); (0, 0) when empty."""
    lib = _lib.load()
    lo, hi = C.c_int64(), C.c_int64()
    st = lib.gpudb_column_minmax(C.c_void_p(col.data_ptr()), col.numel(), col.element_size(), C.byref(lo),
                                 C.byref(hi), C.c_void_p(stream) if stream else None)
    if st != 0:
        raise RuntimeError(f"column_minmax failed: {_lib.last_error(None)}")
    return int(lo.value), int(hi.value)


class MixTables:
    """Resident mixed-workload tables: several mix tables (one Zipf exponent
    each for m_rank_z; m_rank_u is uniform) and one mixdim table, as
    contiguous CUDA tensors, with per-column min / max (zone-map statistics
    computed once at load)."""

    def __init__(self, rows: int, zipf_s: Sequence[float] = (0.8, 0.95, 1.1, 1.3), nranks: int = 1 << 22,
                 dim_rows: int = 1_000_000, seed: int = 20240501, device: str = "cuda", host: bool = False):
        """Generates the tables in HBM with the device generators (values
        identical to the host generators of the same seeds); `host` also
        keeps numpy copies (for the CPU oracle)."""
        import torch
        from . import workloads as W

        self.rows, self.zipf_s, self.nranks, self.dim_rows, self.seed = rows, tuple(zipf_s), nranks, dim_rows, seed
        lib = _lib.load_datagen()
        stream = torch.cuda.current_stream().cuda_stream
        tdt = {np.int32: torch.int32, np.int64: torch.int64}
        self.tables: List[Dict[str, "torch.Tensor"]] = []
        self.host: List[Dict[str, np.ndarray]] = []
        self.stats: List[Dict[str, Tuple[int, int]]] = []
        for t, s in enumerate(self.zipf_s):
            cols = {c: torch.empty(rows, dtype=tdt[dt], device=device) for c, dt in W.MIX_COLUMNS.items()}
            st = lib.gpudb_gen_mix_device(self.table_seed(t), nranks, s, dim_rows, 0, rows,
                                          *(cols[c].data_ptr() for c in W.MIX_COLUMNS), stream)
            if st != 0:
                raise RuntimeError(f"device generator failed: {_lib.datagen_error()}")
            self.stats.append({c: column_minmax(v, stream) for c, v in cols.items()})
            self.tables.append(cols)
            if host:
                self.host.append({c: v.cpu().numpy() for c, v in cols.items()})
        self.dim = {c: torch.empty(dim_rows, dtype=tdt[dt], device=device) for c, dt in W.MIXDIM_COLUMNS.items()}
        if lib.gpudb_gen_mixdim_device(seed, 0, dim_rows, self.dim["md_key"].data_ptr(),
                                       self.dim["md_attr"].data_ptr(), stream) != 0:
            raise RuntimeError(f"device generator failed: {_lib.datagen_error()}")
        self.dim_host = {c: v.cpu().numpy() for c, v in self.dim.items()} if host else None
        self.dim_max_key = dim_rows  # keys are 1..dim_rows
        torch.cuda.synchronize()

    def table_seed(self, t: int) -> int:
        return self.seed + 7919 * t

    def ptr(self, table: int, col: str, row0: int = 0) -> int:
        t = self.tables[table][col]
        return t.data_ptr() + row0 * t.element_size()

    def slice_host(self, q: MixQuery) -> Dict[str, np.ndarray]:
        m = self.host[q.table]
        return {c: a[q.row0:q.row0 + q.rows] for c, a in m.items()}

    def query_struct(self, q: MixQuery, groups: int = 1) -> BatchQueryStruct:
        st = self.stats[q.table]
        kmin, kmax = st[q.key]
        s = BatchQueryStruct(tmpl=TPL[q.tmpl], thr=q.thr, card=max(1, q.card), k=q.k, attr_lt=q.attr_lt,
                             rows=q.rows, key=self.ptr(q.table, q.key, q.row0),
                             filter=self.ptr(q.table, "m_filter", q.row0),
                             value=self.ptr(q.table, "m_value", q.row0),
                             fk=self.ptr(q.table, "m_fk", q.row0),
                             dim_key=self.dim["md_key"].data_ptr(), dim_attr=self.dim["md_attr"].data_ptr(),
                             dim_rows=self.dim_rows, dim_max_key=self.dim_max_key, groups=groups,
                             key_min=kmin, key_max=kmax, filter_min=st["m_filter"][0],
                             filter_max=st["m_filter"][1])
        return s

    def query_array(self, queries: Sequence[MixQuery]) -> np.ndarray:
        """All queries as one array of gpudb_batch_query (groups 1, AUTO
        strategy), built column-wise."""
        n = len(queries)
        a = np.zeros(max(1, n), dtype=QUERY_DTYPE)[:n]
        if n == 0:
            return a
        tb = np.array([q.table for q in queries], dtype=np.int64)
        r0 = np.array([q.row0 for q in queries], dtype=np.int64)
        zipf = np.array([q.key == "m_rank_z" for q in queries])
        a["tmpl"] = [TPL[q.tmpl] for q in queries]
        a["thr"] = [q.thr for q in queries]
        a["card"] = [max(1, q.card) for q in queries]
        a["k"] = [q.k for q in queries]
        a["attr_lt"] = [q.attr_lt for q in queries]
        a["rows"] = [q.rows for q in queries]

        def base(col):
            return np.array([t[col].data_ptr() for t in self.tables], dtype=np.int64)[tb]

        a["key"] = np.where(zipf, base("m_rank_z"), base("m_rank_u")) + 4 * r0
        a["filter"] = base("m_filter") + 4 * r0
        a["value"] = base("m_value") + 8 * r0
        a["fk"] = base("m_fk") + 4 * r0
        a["dim_key"] = self.dim["md_key"].data_ptr()
        a["dim_attr"] = self.dim["md_attr"].data_ptr()
        a["dim_rows"] = self.dim_rows
        a["dim_max_key"] = self.dim_max_key
        a["groups"] = 1
        kmin = np.array([[st["m_rank_u"][0], st["m_rank_z"][0]] for st in self.stats], dtype=np.int64)
        kmax = np.array([[st["m_rank_u"][1], st["m_rank_z"][1]] for st in self.stats], dtype=np.int64)
        a["key_min"] = kmin[tb, zipf.astype(np.int64)]
        a["key_max"] = kmax[tb, zipf.astype(np.int64)]
        a["filter_min"] = np.array([st["m_filter"][0] for st in self.stats])[tb]
        a["filter_max"] = np.array([st["m_filter"][1] for st in self.stats])[tb]
        return a

    def bytes(self) -> int:
        return sum(t.numel() * t.element_size() for tab in self.tables for t in tab.values()) + \
            sum(t.numel() * t.element_size() for t in self.dim.values())


def query_bytes(q: MixQuery, dim_rows: int) -> int:
    """Algorithmic bytes of one query: every referenced column read once
    (the value column of the filtered templates counted in full)."""
    if q.tmpl == "agg":
        return 12 * q.rows
    if q.tmpl == "join":
        return 16 * q.rows + 8 * dim_rows
    return 16 * q.rows


# ---------------------------------------------------------------------------
# pinned result buffers
# ---------------------------------------------------------------------------
class PinnedPool:
    """Pinned host buffers handed out as numpy arrays that own them: when
    the last view of a buffer is dropped it returns to the pool, so batch
    results reach the caller without a host copy and the memory is reused."""

    def __init__(self, alloc=None, free=None):
        lib = None if alloc and free else _lib.load()
        self._alloc = alloc or lib.gpudb_host_alloc
        self._freefn = free or (lambda ptr: lib.gpudb_host_free(C.c_void_p(ptr)))
        self._free: List[Tuple[int, int]] = []  # (bytes, ptr)
        self._lock = threading.Lock()
        self._closed = False

    def array(self, nbytes: int) -> np.ndarray:
        """An int64 array of at least `nbytes` bytes in pinned memory."""
        nbytes = max(64, nbytes)
        with self._lock:
            best = None
            for k, (cap, ptr) in enumerate(self._free):
                if cap >= nbytes and (best is None or cap < self._free[best][0]):
                    best = k
            if best is not None:
                cap, ptr = self._free.pop(best)
            else:
                cap = int(nbytes * 1.25) + 4096
                ptr = self._alloc(cap)
                if not ptr:
                    raise MemoryError(f"pinned host buffer of {cap} bytes")
        buf = (C.c_int64 * (cap // 8)).from_address(ptr)
        weakref.finalize(buf, self._release, cap, ptr)
        return np.ctypeslib.as_array(buf)

    def _release(self, cap: int, ptr: int) -> None:
        with self._lock:
            if self._closed:
                self._freefn(ptr)
            else:
                self._free.append((cap, ptr))

    def close(self) -> None:
        with self._lock:
            self._closed = True
            for _, ptr in self._free:
                self._freefn(ptr)
            self._free.clear()


_POOL: Optional[PinnedPool] = None


def pinned_pool() -> PinnedPool:
    global _POOL
    if _POOL is None:
        _POOL = PinnedPool()
    return _POOL


# ---------------------------------------------------------------------------
# the C batch object
# ---------------------------------------------------------------------------
class Batch:
    """A set of mixed queries on resident device columns (gpudb_batch)."""

    def __init__(self):
        self._lib = _lib.load()
        h = C.c_void_p()
        check(self._lib.gpudb_batch_create(None, C.byref(h)))
        self.handle = h
        self.n = 0

    def close(self) -> None:
        if self.handle:
            self._lib.gpudb_batch_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_queries(self, structs) -> None:
        """Describe the batch: a sequence of BatchQueryStruct, or an array
        of QUERY_DTYPE (MixTables.query_array)."""
        if isinstance(structs, np.ndarray):
            arr = np.ascontiguousarray(structs, dtype=QUERY_DTYPE)
            self._structs = arr
            check(self._lib.gpudb_batch_set_queries(self.handle, arr.ctypes.data if arr.size else None, arr.size))
            self.n = arr.size
            return
        arr = (BatchQueryStruct * max(1, len(structs)))(*structs)
        self._structs = arr
        check(self._lib.gpudb_batch_set_queries(self.handle, arr, len(structs)))
        self.n = len(structs)

    def set_groups(self, i: int, groups: int) -> None:
        check(self._lib.gpudb_batch_set_groups(self.handle, i, int(groups)))

    def set_agg_mode(self, i: int, mode: int) -> None:
        check(self._lib.gpudb_batch_set_agg_mode(self.handle, i, int(mode)))

    def set_tuning(self, block: int = 512, tile_rows: int = 32768, warp_aggregate: bool = True,
                   max_probe: int = 128, group_rows: int = 1, agg_rows: int = 2, shared_warp: int = 1) -> None:
        check(self._lib.gpudb_batch_set_tuning(self.handle, block, tile_rows, int(warp_aggregate), max_probe))
        check(self._lib.gpudb_batch_set_option(self.handle, b"group_rows", group_rows))
        check(self._lib.gpudb_batch_set_option(self.handle, b"agg_rows", agg_rows))
        check(self._lib.gpudb_batch_set_option(self.handle, b"shared_warp", shared_warp))

    def execute(self, use_graph: bool = True) -> Tuple[float, np.ndarray]:
        ms = C.c_double()
        err = np.zeros(max(1, self.n), dtype=np.uint32)
        check(self._lib.gpudb_batch_execute(self.handle, int(use_graph), C.byref(ms), err.ctypes.data))
        return ms.value, err[:self.n]

    def exact_stats(self) -> Tuple[np.ndarray, np.ndarray, float]:
        p = np.zeros(max(1, self.n), dtype=np.uint64)
        d = np.zeros(max(1, self.n), dtype=np.uint64)
        ms = C.c_double()
        check(self._lib.gpudb_batch_exact_stats(self.handle, p.ctypes.data, d.ctypes.data, C.byref(ms)))
        return p[:self.n], d[:self.n], ms.value

    def features(self) -> Tuple[np.ndarray, float]:
        f = np.zeros((max(1, self.n), SIZER_FEATURES), dtype=np.float32)
        ms = C.c_double()
        check(self._lib.gpudb_batch_features(self.handle, f.ctypes.data, C.byref(ms)))
        return f[:self.n], ms.value

    def collect(self) -> Tuple[np.ndarray, np.ndarray, float]:
        """(rows per query, packed int64 rows [total, 3], device+copy ms).
        The packed rows are copied once, by the device, into a pinned buffer
        that the returned array owns (see PinnedPool)."""
        rows = np.zeros(max(1, self.n), dtype=np.uint64)
        need = C.c_uint64()
        ms = C.c_double()
        check(self._lib.gpudb_batch_collect(self.handle, rows.ctypes.data, None, 0, C.byref(need), None))
        host = pinned_pool().array(need.value)
        check(self._lib.gpudb_batch_collect(self.handle, None, host.ctypes.data, host.nbytes, C.byref(need),
                                            C.byref(ms)))
        return rows[:self.n], host[:need.value // 8].reshape(-1, 3), ms.value

    def result_scalar(self, i: int) -> Tuple[int, int]:
        c, lo, hi = C.c_int64(), C.c_uint64(), C.c_int64()
        check(self._lib.gpudb_batch_result_scalar(self.handle, i, C.byref(c), C.byref(lo), C.byref(hi)))
        return c.value, (hi.value << 64) | lo.value

    def result_groups(self, i: int):
        n = C.c_uint64()
        check(self._lib.gpudb_batch_result_groups(self.handle, i, 0, C.byref(n), None, None, None))
        k, c, s = (np.zeros(max(1, n.value), dtype=np.int64) for _ in range(3))
        check(self._lib.gpudb_batch_result_groups(self.handle, i, n.value, C.byref(n), k.ctypes.data,
                                                  c.ctypes.data, s.ctypes.data))
        return k[:n.value], c[:n.value], s[:n.value]

    def result_topk(self, i: int):
        k = np.zeros(16, dtype=np.int64)
        v = np.zeros(16, dtype=np.int64)
        n = C.c_int()
        check(self._lib.gpudb_batch_result_topk(self.handle, i, k.ctypes.data, v.ctypes.data, C.byref(n)))
        return tuple((int(k[j]), int(v[j])) for j in range(n.value))

    def last_launches(self) -> int:
        return int(self._lib.gpudb_batch_last_launches(self.handle))

    STAGES = ("fill", "join_build", "agg_probe", "group", "topk_chunks", "topk_merge")

    def stage_ms(self) -> Dict[str, float]:
        """Per-step device ms of the last execute(use_graph=False)."""
        ms = np.zeros(len(self.STAGES), dtype=np.float64)
        check(self._lib.gpudb_batch_stage_ms(self.handle, ms.ctypes.data))
        return dict(zip(self.STAGES, ms.tolist()))


def unpack_results(queries: Sequence[MixQuery], rows: np.ndarray, packed: np.ndarray,
                   copy: bool = False) -> List[tuple]:
    """Results from gpudb_batch_collect's packed rows (group-by rows as
    "groups_raw" blocks: views into `packed`, which they keep alive, unless
    `copy`)."""
    if copy:
        packed = packed.copy()
    out = []
    off = 0
    for q, r in zip(queries, rows):
        r = int(r)
        blk = packed[off:off + r]
        off += r
        if q.tmpl in ("agg", "join"):
            lo = int(blk[0, 1]) & ((1 << 64) - 1)
            out.append(("scalar", int(blk[0, 0]), (int(blk[0, 2]) << 64) | lo))
        elif q.tmpl == "groupby":
            out.append(("groups_raw", blk))
        else:
            out.append(("topk", tuple((int(a), int(b)) for a, b in blk[:, :2])))
    return out


# ---------------------------------------------------------------------------
# learned sizer
# ---------------------------------------------------------------------------
class Sizer:
    """16 -> 64 -> 64 -> 64 -> 2 MLP (BF16 weights, FP32 accumulate), trained
    and evaluated on the GPU by the library's own kernels."""

    def __init__(self, seed: int = 0, device: int = 0):
        self._lib = _lib.load()
        h = C.c_void_p()
        check(self._lib.gpudb_sizer_create(device, seed, C.byref(h)))
        self.handle = h
        self.nparams = int(self._lib.gpudb_sizer_param_count())
        self._lock = threading.Lock()  # one device workspace: calls from threads take turns

    def close(self) -> None:
        if self.handle:
            self._lib.gpudb_sizer_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def params(self) -> np.ndarray:
        p = np.zeros(self.nparams, dtype=np.float32)
        with self._lock:
            check(self._lib.gpudb_sizer_get_params(self.handle, p.ctypes.data))
        return p

    @params.setter
    def params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.shape == (self.nparams,)
        with self._lock:
            check(self._lib.gpudb_sizer_set_params(self.handle, p.ctypes.data))

    def grads(self, X: np.ndarray, Y: np.ndarray) -> Tuple[np.ndarray, float]:
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.ascontiguousarray(Y, dtype=np.float32)
        g = np.zeros(self.nparams, dtype=np.float32)
        loss = C.c_float()
        with self._lock:
            check(self._lib.gpudb_sizer_grads(self.handle, X.ctypes.data, Y.ctypes.data, X.shape[0], g.ctypes.data,
                                              C.byref(loss)))
        return g, loss.value

    def train(self, X: np.ndarray, Y: np.ndarray, epochs: int = 20, batch: int = 256, lr: float = 2e-3,
              seed: int = 0) -> float:
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.ascontiguousarray(Y, dtype=np.float32)
        loss = C.c_float()
        with self._lock:
            check(self._lib.gpudb_sizer_train(self.handle, X.ctypes.data, Y.ctypes.data, X.shape[0], epochs, batch,
                                              lr, seed, C.byref(loss)))
        return loss.value

    def predict(self, X: np.ndarray) -> np.ndarray:
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.zeros((X.shape[0], SIZER_OUTPUTS), dtype=np.float32)
        if X.shape[0]:
            with self._lock:
                check(self._lib.gpudb_sizer_predict(self.handle, X.ctypes.data, X.shape[0], Y.ctypes.data))
        return Y

    def save(self, path) -> None:
        np.save(path, self.params)

    def load(self, path) -> None:
        self.params = np.load(path)


def labels(queries: Sequence[MixQuery], passing: np.ndarray, distinct: np.ndarray) -> np.ndarray:
    """Sizer targets: (log2(groups + 1) / 24, selectivity)."""
    y = np.zeros((len(queries), SIZER_OUTPUTS), dtype=np.float32)
    for i, q in enumerate(queries):
        y[i, 0] = math.log2(float(distinct[i]) + 1.0) / CARD_SCALE if q.grouped else 0.0
        y[i, 1] = float(passing[i]) / q.rows if q.rows else 0.0
    return y


def groups_from_prediction(q: MixQuery, y0: float, margin: float) -> int:
    """Hash-table sizing from a predicted log2 cardinality, clamped to the
    exact upper bounds (card values of key % card, and the slice rows)."""
    g = (2.0 ** (float(y0) * CARD_SCALE) - 1.0) * margin
    bound = max(1, min(q.card, q.rows))
    return int(min(bound, max(1, math.ceil(g))))


SKEW_SHARE = 0.004           # sample share of the most frequent key that counts as skew


def agg_mode_for(groups: int, features: Optional[np.ndarray], card: Optional[int] = None) -> int:
    """Aggregation strategy of a group-by from its key domain, its expected
    group count and the 4096-row sample (measured on B200, 60M rows: a key
    domain of at most 1024 values indexes the shared table directly; shared
    memory wins for up to ~1K groups and for skewed keys at any
    cardinality, where hot keys would serialise global atomics; the global
    table wins 2-3x for unskewed keys beyond a few thousand groups)."""
    if card is not None and card <= DIRECT_MAX_CARD:
        # ... unless one key holds well above its uniform share: its slot's
        # serialised shared atomics then cost more than warp aggregation
        # (measured, 60M rows: uniform keys 2x faster direct; Zipf(1.1)
        # keys 8-33 % slower)
        skewed = features is not None and features[12] >= max(2.0 / card, DIRECT_SKEW_SHARE)
        return AGG_SHARED if skewed else AGG_SHARED_DIRECT
    if groups <= SHARED_MAX_GROUPS or features is None:
        return AGG_SHARED
    return AGG_SHARED if features[12] >= SKEW_SHARE else AGG_GLOBAL


def sample_estimate(features: np.ndarray) -> np.ndarray:
    """The closed-form sizing estimate the network competes with: the
    uniform-key estimate of feature 14, as log2(groups + 1) / 24."""
    return features[:, 14] * (24.0 / CARD_SCALE)


class ExecutionLog:
    """Features and exact outcomes of executed queries: the sizer's training set."""

    def __init__(self):
        self.X: List[np.ndarray] = []
        self.Y: List[np.ndarray] = []

    def add(self, X: np.ndarray, Y: np.ndarray) -> None:
        self.X.append(np.asarray(X, dtype=np.float32))
        self.Y.append(np.asarray(Y, dtype=np.float32))

    def __len__(self) -> int:
        return sum(x.shape[0] for x in self.X)

    def arrays(self) -> Tuple[np.ndarray, np.ndarray]:
        if not self.X:
            return np.zeros((0, SIZER_FEATURES), np.float32), np.zeros((0, SIZER_OUTPUTS), np.float32)
        return np.concatenate(self.X), np.concatenate(self.Y)

    def save(self, path) -> None:
        X, Y = self.arrays()
        np.savez_compressed(path, X=X, Y=Y)

    @classmethod
    def load(cls, path) -> "ExecutionLog":
        z = np.load(path)
        log = cls()
        log.add(z["X"], z["Y"])
        return log


def log_executions(tables: MixTables, queries: Sequence[MixQuery], log: ExecutionLog,
                   batch_size: int = 1024) -> float:
    """Run the exact statistics pass and the feature sample over `queries`
    (in batches) and append (features, exact outcome) to `log`. Returns the
    device milliseconds spent."""
    ms = 0.0
    b = Batch()
    try:
        for i in range(0, len(queries), batch_size):
            part = list(queries[i:i + batch_size])
            b.set_queries([tables.query_struct(q) for q in part])
            X, t0 = b.features()
            p, d, t1 = b.exact_stats()
            log.add(X, labels(part, p, d))
            ms += t0 + t1
    finally:
        b.close()
    return ms


# ---------------------------------------------------------------------------
# the two execution paths
# ---------------------------------------------------------------------------
class PlainRunner:
    """One query at a time through the engine's generated kernels
    (gpudb_query_run of the mix_* templates), with the exact count pass
    (`distinct` template) sizing every hash table: the plain method, and the
    fallback / judge of the batched path.

    It is the competent per-query form: a query's constants (filter
    threshold, key cardinality, join attribute bound) are kernel arguments
    bound at launch (params=1), so each template compiles once, not once
    per constant set; the context's buffers are reused from query to query
    (they only grow); and a group-by's created groups are compacted on the
    device (compact=1), so collecting its result copies groups x 24 bytes
    rather than the whole table. The count pass still reads its counter on
    the host before the group-by is sized, as the reference's exact sizing
    pass does."""

    SPEC = {"agg": "mix_agg", "join": "mix_join", "groupby": "mix_groupby", "topk": "mix_topk"}

    def __init__(self, ctx, tables: MixTables, tune: str = ""):
        self.ctx, self.tables, self.tune = ctx, tables, tune
        for c, t in tables.dim.items():
            ctx.register_column("mixdim", c, t.data_ptr(), t.numel(), t.element_size())
        self.count_passes = 0
        self.count_s = 0.0  # wall time spent in exact count passes
        self._lock = threading.Lock()  # one engine context: queries from threads take turns
        self._queries = {}

    def _query(self, spec: str):
        q = self._queries.get(spec)
        if q is None:
            q = self._queries[spec] = self.ctx.prepare(spec, self.tune)
        return q

    def _register_slice(self, q: MixQuery) -> None:
        cols = ["m_filter", "m_value"] + (["m_fk"] if q.tmpl == "join" else []) + ([q.key] if q.grouped else [])
        for c in cols:
            t = self.tables.tables[q.table][c]
            self.ctx.register_column("mix", c, t.data_ptr() + q.row0 * t.element_size(), q.rows, t.element_size())
        self.ctx.register_symbol("mix_thr", q.thr)
        if q.grouped:
            self.ctx.register_symbol("mix_card", q.card)
        if q.tmpl == "join":
            self.ctx.register_symbol("mix_attr_lt", q.attr_lt)

    def exact_groups(self, q: MixQuery) -> int:
        t0 = time.perf_counter()
        self._register_slice(q)
        res, _ = self.ctx.run(self._query(f"template=distinct;params=1;key={q.key}"), arrays=True)
        self.count_passes += 1
        self.count_s += time.perf_counter() - t0
        return int(res["distinct"][0])

    def run(self, q: MixQuery) -> tuple:
        with self._lock:
            return self._run(q)

    def _run(self, q: MixQuery) -> tuple:
        self._register_slice(q)
        spec = f"template={self.SPEC[q.tmpl]};params=1"
        if q.grouped:
            groups = self.exact_groups(q)
            self.ctx.register_symbol("mix_groups", max(1, groups))
            spec += f";key={q.key}"
            spec += f";k={q.k}" if q.tmpl == "topk" else ";compact=1"
        if q.tmpl in ("agg", "join"):
            # an exact 128-bit sum: the (small) row form keeps its high word
            res, _ = self.ctx.run(self._query(spec))
            c, s = res.rows[0]
            return ("scalar", int(c), int(s))
        if q.tmpl == "groupby":
            # the compacted groups straight from their device buffers, in
            # table order (a GROUP BY has no row order; `canonical` sorts
            # when a comparison needs it)
            self.ctx.run(self._query(spec), collect=False)
            n = int(self.ctx.read_buffer("mgc_n", np.uint64, 1)[0])
            # into fresh host arrays (pooled pinned buffers measured no
            # faster here, and the callers keep hundreds of answers alive,
            # so a pool would keep page-locking more memory)
            return ("groups_cols",) + tuple(self.ctx.read_buffer(name, np.int64, n)
                                            for name in ("mgc_key", "mgc_count", "mgc_sum"))
        res, _ = self.ctx.run(self._query(spec), arrays=True)
        return ("topk", tuple((int(k), int(v)) for k, v in zip(res["key"], res["sum"])))


@dataclass
class BatchReport:
    sizing: str
    queries: int
    features_ms: float = 0.0
    predict_ms: float = 0.0
    stats_ms: float = 0.0
    execute_ms: float = 0.0
    collect_ms: float = 0.0
    plan_ms: float = 0.0     # host: describing the batch (arena plan, descriptor upload)
    unpack_ms: float = 0.0   # host: turning the collected rows into per-query results
    overflowed: List[int] = field(default_factory=list)
    fallback_s: float = 0.0
    wall_s: float = 0.0
    table_slots: int = 0
    launches: int = 0
    result_bytes: int = 0


class BatchRunner:
    """The batched form: all queries of a batch through the persistent
    work-queue kernels, hash tables sized by `sizing`:
      "learned" — the sizer's predicted cardinality (no count pass);
      "exact"   — the batched exact count pass;
      "bound"   — the exact upper bound min(card, rows) (no pass, largest tables).
    Queries whose table overflowed re-run through the plain exact path."""

    def __init__(self, tables: MixTables, sizing: str = "learned", sizer: Optional[Sizer] = None,
                 plain: Optional[PlainRunner] = None, margin: float = 1.5, use_graph: bool = True,
                 tuning: Optional[dict] = None, agg_mode: Optional[int] = None):
        if sizing == "learned" and sizer is None:
            raise ValueError("learned sizing needs a trained Sizer")
        self.tables, self.sizing, self.sizer, self.plain = tables, sizing, sizer, plain
        self.margin, self.use_graph, self.agg_mode = margin, use_graph, agg_mode
        self.batch = Batch()
        if tuning:
            self.batch.set_tuning(**tuning)
        self._key = None
        self._groups = None
        self._features = None

    def close(self) -> None:
        self.batch.close()

    def size(self, queries: Sequence[MixQuery], report: BatchReport) -> List[int]:
        b = self.batch
        if self.sizing == "learned":
            X, report.features_ms = b.features()
            self._features = X
            t = time.perf_counter()
            Y = self.sizer.predict(X)
            report.predict_ms = 1e3 * (time.perf_counter() - t)
            return [groups_from_prediction(q, Y[i, 0], self.margin) if q.grouped else 1
                    for i, q in enumerate(queries)]
        if self.sizing == "exact":
            _, d, report.stats_ms = b.exact_stats()
            return [max(1, int(d[i])) if q.grouped else 1 for i, q in enumerate(queries)]
        if self.sizing == "bound":
            return [max(1, min(q.card, q.rows)) if q.grouped else 1 for q in queries]
        raise ValueError(f"unknown sizing '{self.sizing}'")

    def run(self, queries: Sequence[MixQuery], copy: bool = False) -> Tuple[List[tuple], BatchReport]:
        """Results of group-by queries are "groups_raw" blocks: views of the
        pinned buffer the device wrote them into (it returns to the pool once
        no view is left), or private copies with copy=True."""
        t0 = time.perf_counter()
        report = BatchReport(self.sizing, len(queries))
        key = tuple(queries)
        b = self.batch
        tp = time.perf_counter()
        if key != self._key:
            self._arr = self.tables.query_array(queries)
            b.set_queries(self._arr)
            self._key, self._groups = key, None
        report.plan_ms = (time.perf_counter() - tp) * 1e3
        self._features = None
        groups = self.size(queries, report)
        modes = [(self.agg_mode if self.agg_mode is not None else
                  agg_mode_for(g, None if self._features is None else self._features[i], q.card))
                 if q.grouped else AGG_AUTO
                 for i, (g, q) in enumerate(zip(groups, queries))]
        if (groups, modes) != self._groups:
            tp = time.perf_counter()
            self._arr["groups"] = groups
            self._arr["agg_mode"] = modes
            b.set_queries(self._arr)  # one call re-plans the arena
            self._groups = (groups, modes)
            report.plan_ms += (time.perf_counter() - tp) * 1e3
        report.table_slots = sum(1 << max(4, math.ceil(math.log2(2 * g))) for g, q in zip(groups, queries)
                                 if q.grouped)
        report.execute_ms, err = b.execute(self.use_graph)
        report.launches = b.last_launches()
        rows, packed, report.collect_ms = b.collect()
        report.result_bytes = int(packed.nbytes)
        tu = time.perf_counter()
        results = unpack_results(queries, rows, packed, copy=copy)
        report.unpack_ms = (time.perf_counter() - tu) * 1e3
        err = [int(e) for e in err]
        bad = [i for i, e in enumerate(err) if e & DEVERR_HASH_OVERFLOW]
        other = [i for i, e in enumerate(err) if e & ~DEVERR_HASH_OVERFLOW]
        if other:
            raise RuntimeError(f"device errors {[(i, int(err[i])) for i in other[:8]]}")
        if bad:
            if self.plain is None:
                raise RuntimeError(f"{len(bad)} hash tables overflowed and no exact fallback is configured")
            tf = time.perf_counter()
            for i in bad:
                results[i] = self.plain.run(queries[i])
            report.fallback_s = time.perf_counter() - tf
        report.overflowed = bad
        report.wall_s = time.perf_counter() - t0
        return results, report


def train_sizer(log: ExecutionLog, seed: int = 0, epochs: int = 30, batch: int = 512, lr: float = 2e-3,
                holdout: float = 0.1) -> Tuple[Sizer, dict]:
    """Train a sizer on an execution log; report held-out errors of the
    network and of the closed-form sample estimate."""
    X, Y = log.arrays()
    rng = np.random.default_rng(seed)
    idx = rng.permutation(X.shape[0])
    nh = max(1, int(holdout * X.shape[0]))
    te, tr = idx[:nh], idx[nh:]
    s = Sizer(seed=seed)
    t = time.perf_counter()
    loss = s.train(X[tr], Y[tr], epochs=epochs, batch=batch, lr=lr, seed=seed)
    train_s = time.perf_counter() - t
    P = s.predict(X[te])
    grouped = X[te, 2] + X[te, 3] > 0
    err_net = np.abs(P[grouped, 0] - Y[te][grouped, 0]) * CARD_SCALE
    err_est = np.abs(sample_estimate(X[te][grouped]) - Y[te][grouped, 0]) * CARD_SCALE
    return s, {"train_loss": loss, "train_s": train_s, "train_rows": int(tr.size), "holdout_rows": int(te.size),
               "log2_err_net_mean": float(err_net.mean()) if err_net.size else 0.0,
               "log2_err_net_p99": float(np.quantile(err_net, 0.99)) if err_net.size else 0.0,
               "log2_err_estimate_mean": float(err_est.mean()) if err_est.size else 0.0,
               "log2_err_estimate_p99": float(np.quantile(err_est, 0.99)) if err_est.size else 0.0,
               "sel_err_net_mean": float(np.abs(P[:, 1] - Y[te][:, 1]).mean())}
