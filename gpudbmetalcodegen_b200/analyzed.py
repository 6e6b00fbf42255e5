"""Analyzed queries through the C-ABI (include/gpudb_engine.h, gpudb_aq_*).

The reference plans from an AnalyzedQuery (codegen/planning/query_plan.h:
14-183, query_analyzer.h:14-81) with buildMetalPlan(aq, name)
(metal_plan_builder.cpp:2035-2109). ``AnalyzedQuery`` here builds the same
structure node by node — expressions, predicates, aggregate targets, GROUP
BY, ORDER BY, LIMIT — and ``prepare`` plans it with
gpudb_query_prepare_analyzed. Nodes are opaque handles owned by their
query. Errors raise GpudbError with the planner's reason.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

from . import _lib
from ._lib import GpudbError, check

ADD, SUB, MUL, DIV = range(4)
EQ, NE, LT, LE, GT, GE = range(6)
SUM, COUNT, AVG, MIN, MAX = range(5)


class AnalyzedQuery:
    def __init__(self):
        self._lib = _lib.load()
        h = C.c_void_p()
        check(self._lib.gpudb_aq_create(C.byref(h)))
        self.handle = h

    def _node(self, p):
        if not p:
            raise GpudbError(-1, "analyzed query: invalid node or argument")
        return p

    # ---- expressions (Expr::col / lit / litf / lits / binary) ----------
    def col(self, table: str, column: str):
        return self._node(self._lib.gpudb_aq_col(self.handle, table.encode(), column.encode()))

    def ref(self, alias: str):
        """A select target's alias (ORDER BY revenue)."""
        return self._node(self._lib.gpudb_aq_col(self.handle, b"", alias.encode()))

    def lit(self, v: int):
        return self._node(self._lib.gpudb_aq_lit_int(self.handle, int(v)))

    def litf(self, v: float):
        return self._node(self._lib.gpudb_aq_lit_decimal(self.handle, float(v)))

    def lits(self, v: str):
        return self._node(self._lib.gpudb_aq_lit_str(self.handle, v.encode()))

    def binary(self, op: int, left, right):
        return self._node(self._lib.gpudb_aq_binary(self.handle, op, left, right))

    # ---- predicates ------------------------------------------------------
    def cmp(self, op: int, left, right):
        return self._node(self._lib.gpudb_aq_cmp(self.handle, op, left, right))

    def between(self, e, lo, hi):
        return self._node(self._lib.gpudb_aq_between(self.handle, e, lo, hi))

    def in_list(self, e, values: Sequence):
        arr = (C.c_void_p * max(1, len(values)))(*values)
        return self._node(self._lib.gpudb_aq_in_list(self.handle, e, arr, len(values)))

    def and_(self, *children):
        arr = (C.c_void_p * max(1, len(children)))(*children)
        return self._node(self._lib.gpudb_aq_and(self.handle, arr, len(children)))

    def or_(self, *children):
        arr = (C.c_void_p * max(1, len(children)))(*children)
        return self._node(self._lib.gpudb_aq_or(self.handle, arr, len(children)))

    def not_(self, child):
        return self._node(self._lib.gpudb_aq_not(self.handle, child))

    # ---- the query's fields ---------------------------------------------
    def table(self, name: str) -> "AnalyzedQuery":
        check(self._lib.gpudb_aq_add_table(self.handle, name.encode()))
        return self

    def join(self, left_table: str, left_col: str, right_table: str, right_col: str) -> "AnalyzedQuery":
        check(self._lib.gpudb_aq_add_join(self.handle, left_table.encode(), left_col.encode(), right_table.encode(),
                                          right_col.encode()))
        return self

    def filter(self, pred) -> "AnalyzedQuery":
        check(self._lib.gpudb_aq_add_filter(self.handle, pred))
        return self

    def target(self, e, alias: str = "") -> "AnalyzedQuery":
        check(self._lib.gpudb_aq_add_target(self.handle, e, alias.encode()))
        return self

    def agg(self, func: int, e, alias: str) -> "AnalyzedQuery":
        check(self._lib.gpudb_aq_add_agg(self.handle, func, e, alias.encode()))
        return self

    def group_by(self, e) -> "AnalyzedQuery":
        check(self._lib.gpudb_aq_add_group_by(self.handle, e))
        return self

    def order_by(self, e, descending: bool = False) -> "AnalyzedQuery":
        check(self._lib.gpudb_aq_add_order_by(self.handle, e, 1 if descending else 0))
        return self

    def limit(self, n: int) -> "AnalyzedQuery":
        check(self._lib.gpudb_aq_set_limit(self.handle, n))
        return self

    # ---- lowering / planning ---------------------------------------------
    def lower(self, expr) -> tuple:
        """(CUDA expression, decimal scale) of an expression node."""
        buf = C.create_string_buffer(4096)
        sc = C.c_int()
        check(self._lib.gpudb_aq_lower_expr(expr, buf, 4096, C.byref(sc)))
        return buf.value.decode(), sc.value

    def lower_pred(self, pred) -> str:
        buf = C.create_string_buffer(4096)
        check(self._lib.gpudb_aq_lower_pred(pred, buf, 4096))
        return buf.value.decode()

    def prepare(self, ctx=None, name: str = "", tune: str = ""):
        from .engine import Query
        h = C.c_void_p()
        st = self._lib.gpudb_query_prepare_analyzed(ctx.handle if ctx else None, self.handle, name.encode(),
                                                    tune.encode(), C.byref(h))
        check(st, ctx.handle if ctx else None)
        return Query(f"analyzed={name}", tune, ctx, handle=h)

    def close(self) -> None:
        if self.handle:
            self._lib.gpudb_aq_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
