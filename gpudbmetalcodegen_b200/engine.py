"""Python host layer over the C-ABI (include/gpudb_rt.h, gpudb_engine.h).

Mirrors the reference's host objects one for one:
  * ``Context``  — MetalGenericExecutor (register tables/symbols/scalars,
    execute, read buffers, release) + the runCodegenQuery flow;
  * ``Query``    — a prepared plan: buildMetalPlan + generateFromPlan +
    RuntimeCompiler (source, plan description, compile log);
  * ``Result``   — GenericResult (columns, rows, toCanonical);
  * ``compare_canonical`` — the golden check of ``--check``.
Errors raise ``GpudbError`` carrying the C status and the context's message,
as the reference surfaces nullptr/exceptions (runtime_compiler.cpp:28-40,
metal_generic_executor.cpp:91-93).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Any, Dict, Iterable, List, Mapping, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import GpudbError, check, get_string

NP_ELEM = {np.dtype(np.int32): 4, np.dtype(np.int64): 8, np.dtype(np.uint8): 1, np.dtype(np.uint32): 4,
           np.dtype(np.uint64): 8, np.dtype(np.float64): 8, np.dtype(np.int8): 1}


@dataclass
class Timing:
    total_ms: float
    phase_ms: List[float]
    phase_grid: List[int]
    phase_block: List[int]
    device_error: int
    launches: int
    alloc_ms: float = 0.0
    plan_ms: float = 0.0
    codegen_ms: float = 0.0
    compile_ms: float = 0.0
    collect_ms: float = 0.0

    @staticmethod
    def from_c(t: _lib.Timing) -> "Timing":
        n = t.nphases
        return Timing(t.total_ms, list(t.phase_ms[:n]), list(t.phase_grid[:n]), list(t.phase_block[:n]),
                      t.device_error, t.launches, t.alloc_ms, t.plan_ms, t.codegen_ms, t.compile_ms, t.collect_ms)


@dataclass
class Result:
    """GenericResult: named typed columns and rows of Python values."""
    columns: List[str]
    types: List[str]
    rows: List[tuple]
    canonical: str = ""
    exact: str = ""

    def column(self, name: str) -> List[Any]:
        i = self.columns.index(name)
        return [r[i] for r in self.rows]

    def as_dicts(self) -> List[Dict[str, Any]]:
        return [dict(zip(self.columns, r)) for r in self.rows]


def _result_from_c(res) -> Result:
    lib = _lib.load()
    nc, nr = C.c_int(), C.c_longlong()
    lib.gpudb_result_shape(res, C.byref(nc), C.byref(nr))
    names, types = [], []
    for c in range(nc.value):
        buf = C.create_string_buffer(256)
        t = C.c_int()
        lib.gpudb_result_column(res, c, buf, 256, C.byref(t))
        names.append(buf.value.decode())
        types.append({0: "int", 1: "double", 2: "string"}[t.value])
    cols: List[List[Any]] = []
    for c, t in enumerate(types):
        if t == "int":
            out = np.zeros(nr.value, dtype=np.int64)
            if lib.gpudb_result_export_i64(res, c, out.ctypes.data, nr.value) == 0:
                cols.append([int(v) for v in out])
                continue
            vals = []
            lo, hi = C.c_int64(), C.c_int64()
            for r in range(nr.value):
                lib.gpudb_result_get_int(res, r, c, C.byref(lo), C.byref(hi))
                vals.append((hi.value << 64) | (lo.value & 0xFFFFFFFFFFFFFFFF))
            cols.append(vals)
        elif t == "double":
            v = C.c_double()
            vals = []
            for r in range(nr.value):
                lib.gpudb_result_get_f64(res, r, c, C.byref(v))
                vals.append(v.value)
            cols.append(vals)
        else:
            vals = []
            for r in range(nr.value):
                buf = C.create_string_buffer(256)
                lib.gpudb_result_get_str(res, r, c, buf, 256)
                vals.append(buf.value.decode())
            cols.append(vals)
    rows = list(zip(*cols)) if cols else []
    canonical = get_string(lib.gpudb_result_canonical, res, 0) if nr.value <= 100000 else ""
    exact = get_string(lib.gpudb_result_canonical, res, 1) if nr.value <= 100000 else ""
    return Result(names, types, rows, canonical, exact)


def _arrays_from_c(res) -> Dict[str, np.ndarray]:
    """Integer result columns as numpy int64 arrays (one bulk export per
    column, no per-row Python objects) — for large results."""
    lib = _lib.load()
    nc, nr = C.c_int(), C.c_longlong()
    lib.gpudb_result_shape(res, C.byref(nc), C.byref(nr))
    out = {}
    for c in range(nc.value):
        buf = C.create_string_buffer(256)
        t = C.c_int()
        lib.gpudb_result_column(res, c, buf, 256, C.byref(t))
        if t.value != 0:
            continue
        a = np.zeros(nr.value, dtype=np.int64)
        check(lib.gpudb_result_export_i64(res, c, a.ctypes.data, nr.value))
        out[buf.value.decode()] = a
    return out


class Query:
    """A planned + generated (+ compiled) query."""

    def __init__(self, spec: str, tune: str = "", ctx: Optional["Context"] = None, handle=None):
        self._lib = _lib.load()
        self.spec = spec
        self.tune = tune
        self.ctx = ctx
        if handle is not None:  # prepared elsewhere (an analyzed query)
            self.handle = handle
            return
        h = C.c_void_p()
        st = self._lib.gpudb_query_prepare(ctx.handle if ctx else None, spec.encode(), tune.encode(), C.byref(h))
        check(st, ctx.handle if ctx else None)
        self.handle = h

    @property
    def source(self) -> str:
        return get_string(self._lib.gpudb_query_source, self.handle)

    @property
    def plan(self) -> str:
        return get_string(self._lib.gpudb_query_describe, self.handle)

    @property
    def compile_log(self) -> str:
        return get_string(self._lib.gpudb_query_compile_log, self.handle)

    def close(self) -> None:
        if self.handle:
            self._lib.gpudb_query_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Context:
    """One execution context on one GPU (not thread-safe; one per thread)."""

    def __init__(self, device: int = 0):
        self._lib = _lib.load()
        h = C.c_void_p()
        check(self._lib.gpudb_create(device, C.byref(h)), None)
        self.handle = h
        self._queries: Dict[tuple, Query] = {}
        self._keep: List[Any] = []
        self._table_rows: Dict[str, int] = {}
        self._tune_cache = None

    # ---- lifetime ---------------------------------------------------------
    def close(self) -> None:
        for q in self._queries.values():
            q.close()
        self._queries.clear()
        if self.handle:
            self._lib.gpudb_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- device info --------------------------------------------------------
    def device_info(self) -> Dict[str, int]:
        sms, ma, mi = C.c_int(), C.c_int(), C.c_int()
        check(self._lib.gpudb_device_info(self.handle, C.byref(sms), C.byref(ma), C.byref(mi)), self.handle)
        return {"num_sms": sms.value, "cc_major": ma.value, "cc_minor": mi.value}

    @property
    def stream_ptr(self) -> int:
        return int(self._lib.gpudb_stream(self.handle) or 0)

    def synchronize(self) -> None:
        check(self._lib.gpudb_synchronize(self.handle), self.handle)

    # ---- registration (MetalGenericExecutor::register*) ------------------------
    def register_column(self, table: str, column: str, dptr: int, rows: int, elem_bytes: int) -> None:
        check(self._lib.gpudb_register_column(self.handle, table.encode(), column.encode(), C.c_void_p(dptr), rows,
                                              elem_bytes), self.handle)
        self._table_rows[table] = rows

    def register_tensor(self, table: str, column: str, t) -> None:
        """Register a contiguous CUDA torch tensor as a resident column."""
        if not t.is_cuda or not t.is_contiguous():
            raise ValueError("register_tensor needs a contiguous CUDA tensor")
        self._keep.append(t)
        self.register_column(table, column, t.data_ptr(), t.numel(), t.element_size())

    def run_sql(self, sql: str, tune: str = "", collect: bool = True) -> tuple:
        """Run a SELECT through the template its shape maps to (sql_to_spec)."""
        return self.run(sql_to_spec(sql), tune, collect=collect)

    def load_colbin(self, path: str, table: str, specs) -> None:
        """Upload columns of a .colbin v2 file into resident HBM as `table`'s
        columns. `specs`: (source field index, engine column, transform,
        scale) tuples, transform one of _lib.COLBIN_AS_IS / WIDEN / DECIMAL
        / DAYS."""
        arr = (_lib.ColbinLoadSpec * len(specs))()
        names = [c.encode() for _, c, _, _ in specs]
        for k, (idx, _, tr, sc) in enumerate(specs):
            arr[k] = _lib.ColbinLoadSpec(idx, names[k], tr, sc)
        check(self._lib.gpudb_colbin_load(self.handle, path.encode(), table.encode(), arr, len(specs)), self.handle)
        rows = colbin_inspect(path)["rows"]
        self._table_rows[table] = rows

    def register_host_column(self, table: str, column: str, host_ptr: int, rows: int, elem_bytes: int) -> None:
        """A pinned host column (gpudb_host_alloc) read in place by kernels
        that materialise it late; see gpudb_register_host_column."""
        check(self._lib.gpudb_register_host_column(self.handle, table.encode(), column.encode(), C.c_void_p(host_ptr),
                                                   rows, elem_bytes), self.handle)

    def upload_column(self, table: str, column: str, arr: np.ndarray) -> None:
        arr = np.ascontiguousarray(arr)
        check(self._lib.gpudb_upload_column(self.handle, table.encode(), column.encode(), arr.ctypes.data,
                                            arr.shape[0], NP_ELEM[arr.dtype]), self.handle)
        self._table_rows[table] = arr.shape[0]
        # the copy is stream-ordered: keep the host array alive until it completed
        self.synchronize()

    def upload_table(self, table: str, columns: Mapping[str, np.ndarray]) -> None:
        for name, arr in columns.items():
            self.upload_column(table, name, arr)

    def register_rows(self, table: str, rows: int) -> None:
        check(self._lib.gpudb_register_rows(self.handle, table.encode(), rows), self.handle)

    def register_symbol(self, name: str, value: int) -> None:
        check(self._lib.gpudb_register_symbol(self.handle, name.encode(), int(value)), self.handle)

    def get_symbol(self, name: str) -> int:
        v = C.c_uint64()
        check(self._lib.gpudb_get_symbol(self.handle, name.encode(), C.byref(v)), self.handle)
        return v.value

    def register_scalar(self, name: str, value) -> None:
        if isinstance(value, float):
            check(self._lib.gpudb_register_scalar_f64(self.handle, name.encode(), value), self.handle)
        else:
            check(self._lib.gpudb_register_scalar_i64(self.handle, name.encode(), int(value)), self.handle)

    def register_max_key(self, column: str) -> int:
        v = C.c_longlong()
        check(self._lib.gpudb_register_max_key(self.handle, column.encode(), C.byref(v)), self.handle)
        return v.value

    def set_use_graphs(self, on: bool) -> None:
        check(self._lib.gpudb_set_use_graphs(self.handle, int(on)), self.handle)

    # ---- queries -------------------------------------------------------------
    def largest_table_rows(self) -> int:
        return max(self._table_rows.values(), default=0)

    def resolve_tune(self, spec: str, tune: str) -> str:
        """tune="auto": the autotuner's stored choice for this template at the
        size of the largest registered table ("" when none is stored)."""
        if tune != "auto":
            return tune
        from .autotune import TuneCache
        if self._tune_cache is None:
            self._tune_cache = TuneCache()
        template = dict(kv.split("=", 1) for kv in spec.split(";") if "=" in kv).get("template", "")
        return self._tune_cache.get(template, self.largest_table_rows()) or ""

    def prepare(self, spec: str, tune: str = "") -> Query:
        tune = self.resolve_tune(spec, tune)
        key = (spec, tune)
        q = self._queries.get(key)
        if q is None:
            q = Query(spec, tune, self)
            self._queries[key] = q
        return q

    def run(self, spec_or_query, tune: str = "", warmup: int = 0, measured: int = 1,
            collect: bool = True, arrays: bool = False) -> tuple:
        """Plan/compile (cached), size, execute, collect. Returns (Result|None, Timing);
        with arrays=True the result is a dict of int64 numpy columns instead."""
        q = spec_or_query if isinstance(spec_or_query, Query) else self.prepare(spec_or_query, tune)
        res = C.c_void_p()
        t = _lib.Timing()
        st = self._lib.gpudb_query_run(self.handle, q.handle, warmup, measured,
                                       C.byref(res) if collect else None, C.byref(t))
        timing = Timing.from_c(t)
        if st != 0:
            err = GpudbError(st, _lib.last_error(self.handle))
            err.timing = timing  # type: ignore[attr-defined]
            raise err
        out = None
        if collect:
            try:
                out = _arrays_from_c(res) if arrays else _result_from_c(res)
            finally:
                self._lib.gpudb_result_free(res)
        return out, timing

    def run_streamed(self, spec_or_query, table: str, columns: Sequence[tuple], rows: int, chunk_rows: int,
                     tune: str = "", collect: bool = True, arrays: bool = False) -> tuple:
        """Chunked streaming run of a query whose scans of `table` read it
        from host memory: `columns` are (column, host pointer, element
        bytes, in_place) tuples over pinned host memory (in_place columns
        stay on the host and are read over the link by the rows that reach
        them; the rest are copied a chunk at a time, overlapping the
        kernels of earlier chunks). Returns (Result|None, Timing)."""
        q = spec_or_query if isinstance(spec_or_query, Query) else self.prepare(spec_or_query, tune)
        cols = (_lib.StreamColumn * max(1, len(columns)))()
        keep = []
        for i, (name, ptr, elem, in_place) in enumerate(columns):
            keep.append(name.encode())
            cols[i] = _lib.StreamColumn(keep[-1], C.c_void_p(ptr), int(elem), int(bool(in_place)))
        res = C.c_void_p()
        t = _lib.Timing()
        st = self._lib.gpudb_query_run_streamed(self.handle, q.handle, table.encode(), cols, len(columns), rows,
                                                chunk_rows, C.byref(res) if collect else None, C.byref(t))
        timing = Timing.from_c(t)
        if st != 0:
            raise GpudbError(st, _lib.last_error(self.handle))
        out = None
        if collect:
            try:
                out = _arrays_from_c(res) if arrays else _result_from_c(res)
            finally:
                self._lib.gpudb_result_free(res)
        return out, timing

    def collect(self, query: "Query") -> Result:
        """The result the last execution of `query` left in the buffers
        (e.g. the last of many enqueued graph replays), without running it."""
        res = C.c_void_p()
        check(self._lib.gpudb_query_collect(self.handle, query.handle, C.byref(res)), self.handle)
        try:
            return _result_from_c(res)
        finally:
            self._lib.gpudb_result_free(res)

    def enqueue(self, spec_or_query, tune: str = "") -> None:
        """Enqueue one execution and return without waiting (no timing, no
        result). Device errors surface at the next sync() or run()."""
        q = spec_or_query if isinstance(spec_or_query, Query) else self.prepare(spec_or_query, tune)
        check(self._lib.gpudb_query_enqueue(self.handle, q.handle), self.handle)

    def sync(self) -> None:
        """Wait for enqueued executions; raises GpudbError (status
        GPUDB_E_DEVICE, `device_error` set) if any raised a device error."""
        bits = C.c_uint()
        st = self._lib.gpudb_ctx_sync(self.handle, C.byref(bits))
        if st != 0:
            err = GpudbError(st, _lib.last_error(self.handle))
            err.device_error = bits.value  # type: ignore[attr-defined]
            raise err

    def algorithmic_bytes(self, query: Query) -> int:
        v = C.c_longlong()
        check(self._lib.gpudb_query_algorithmic_bytes(self.handle, query.handle, C.byref(v)), self.handle)
        return v.value

    def read_buffer(self, name: str, dtype, count: int, out: Optional[np.ndarray] = None) -> np.ndarray:
        """The first `count` elements of device buffer `name`; into `out`
        (a C-contiguous array of that dtype, e.g. a view of pinned memory)
        when given."""
        if out is None:
            out = np.empty(count, dtype=dtype)
        elif out.dtype != np.dtype(dtype) or out.size < count or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous array of the buffer's dtype with room for count elements")
        out = out[:count]
        check(self._lib.gpudb_read_buffer(self.handle, name.encode(), out.ctypes.data, out.nbytes), self.handle)
        return out

    def release_buffers(self) -> None:
        check(self._lib.gpudb_release_buffers(self.handle), self.handle)


def compare_canonical(got: str, expected: str, abs_tol: float = 1e-2, rel_tol: float = 1e-4) -> str:
    """'' on match, else the first mismatch (reference --check semantics)."""
    lib = _lib.load()
    buf = C.create_string_buffer(1024)
    ok = lib.gpudb_compare_canonical(got.encode(), expected.encode(), abs_tol, rel_tol, buf, 1024)
    return "" if ok else buf.value.decode()


def compile_check(source: str) -> tuple:
    """NVRTC compile-only for sm_100a (no GPU). Returns (ok, log, ms)."""
    lib = _lib.load()
    buf = C.create_string_buffer(1 << 20)
    ms = C.c_double()
    st = lib.gpudb_compile_check(source.encode(), buf, 1 << 20, C.byref(ms))
    return st == 0, buf.value.decode(errors="replace"), ms.value


def templates() -> List[str]:
    return get_string(_lib.load().gpudb_list_templates).split(",")


def colbin_inspect(path: str) -> dict:
    """Header and column directory of a .colbin v2 file (no GPU needed)."""
    lib = _lib.load()
    rows, n = C.c_uint64(), C.c_uint32()
    cols = (_lib.ColbinColumn * 256)()
    check(lib.gpudb_colbin_inspect(path.encode(), C.byref(rows), C.byref(n), cols, 256))
    return {"rows": rows.value, "columns": [{"index": c.column_index, "dtype": c.dtype, "fixed_width": c.fixed_width,
                                               "offset": c.offset, "size_bytes": c.size_bytes}
                                              for c in cols[:min(n.value, 256)]]}


def sql_to_spec(sql: str) -> str:
    """The pipeline-template spec of a SELECT over the engine's tables
    (no GPU needed); raises GpudbError naming what does not map."""
    buf = C.create_string_buffer(1024)
    check(_lib.load().gpudb_sql_to_spec(sql.encode(), buf, 1024))
    return buf.value.decode()
