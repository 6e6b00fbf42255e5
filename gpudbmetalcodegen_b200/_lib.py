"""ctypes bindings for libgpudb.so (include/gpudb_rt.h, gpudb_engine.h,
gpudb_batch.h) and for the data generators' own library libgpudb_datagen.so
(include/gpudb_datagen.h).

Both are built in-tree by ``build_native.build()``. Loading fails loudly
when a library is missing: there is no Python or CPU fallback for any
operation of the engine.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libgpudb.so"
DATAGEN_PATH = Path(__file__).resolve().parent / "lib" / "libgpudb_datagen.so"

GPUDB_OK = 0
STATUS_NAMES = {0: "OK", -1: "INVALID", -2: "PLAN", -3: "ALLOC", -4: "LAUNCH", -5: "COMPILE", -6: "CUDA",
                -7: "DEVICE", -8: "NOGPU"}
DEVERR_HASH_OVERFLOW = 0x1
DEVERR_WAIT_TIMEOUT = 0x2
DEVERR_BOUNDS = 0x4
DEVERR_SENTINEL_KEY = 0x8
DEVERR_CAPACITY = 0x10

PARAM_TABLE_DATA, PARAM_TABLE_SIZE, PARAM_DEVICE_BUFFER, PARAM_CONSTANT_SCALAR, PARAM_CONSTANT_DATA, \
    PARAM_ERROR_WORD, PARAM_BUFFER_LENGTH = range(7)
COL_INT, COL_DOUBLE, COL_STRING = 0, 1, 2
MAX_PHASES = 32


class BindingDesc(C.Structure):
    _fields_ = [("name", C.c_char_p), ("kind", C.c_int), ("elem_type", C.c_char_p), ("table", C.c_char_p),
                ("size_expr", C.c_char_p), ("zero_init", C.c_int), ("fill_byte", C.c_int), ("read_only", C.c_int)]


class PhaseDesc(C.Structure):
    _fields_ = [("name", C.c_char_p), ("scanned_table", C.c_char_p), ("block_size", C.c_int),
                ("max_blocks", C.c_int), ("single_thread", C.c_int), ("dynamic_smem_bytes", C.c_int),
                ("tile_rows", C.c_int), ("rows_per_thread", C.c_int), ("bindings", C.POINTER(BindingDesc)),
                ("nbindings", C.c_int)]


class StreamColumn(C.Structure):
    _fields_ = [("column", C.c_char_p), ("host", C.c_void_p), ("elem_bytes", C.c_int32), ("in_place", C.c_int32)]


class Timing(C.Structure):
    _fields_ = [("total_ms", C.c_double), ("nphases", C.c_int), ("phase_ms", C.c_double * MAX_PHASES),
                ("phase_grid", C.c_int * MAX_PHASES), ("phase_block", C.c_int * MAX_PHASES),
                ("device_error", C.c_uint), ("launches", C.c_longlong), ("alloc_ms", C.c_double),
                ("plan_ms", C.c_double), ("codegen_ms", C.c_double), ("compile_ms", C.c_double),
                ("collect_ms", C.c_double)]


class ColbinColumn(C.Structure):
    _fields_ = [("column_index", C.c_int32), ("dtype", C.c_uint8), ("fixed_width", C.c_uint16),
                ("offset", C.c_uint64), ("size_bytes", C.c_uint64)]


class ColbinLoadSpec(C.Structure):
    _fields_ = [("column_index", C.c_int32), ("column", C.c_char_p), ("transform", C.c_int32), ("scale", C.c_int32)]


COLBIN_AS_IS, COLBIN_WIDEN, COLBIN_DECIMAL, COLBIN_DAYS = 0, 1, 2, 3


# (name, restype, argtypes) for every exported entry point.
_SIGNATURES = [
    # gpudb_rt.h
    ("gpudb_create", C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    ("gpudb_destroy", None, [C.c_void_p]),
    ("gpudb_last_error", C.c_size_t, [C.c_void_p, C.c_char_p, C.c_size_t]),
    ("gpudb_stream", C.c_void_p, [C.c_void_p]),
    ("gpudb_device_info", C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    ("gpudb_synchronize", C.c_int, [C.c_void_p]),
    ("gpudb_compile", C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(C.c_char_p), C.c_int, C.POINTER(C.c_void_p)]),
    ("gpudb_module_free", None, [C.c_void_p]),
    ("gpudb_compile_check", C.c_int, [C.c_char_p, C.c_char_p, C.c_size_t, C.POINTER(C.c_double)]),
    ("gpudb_set_fast_math", None, [C.c_int]),
    ("gpudb_set_kernel_cache_dir", None, [C.c_char_p]),
    ("gpudb_register_column", C.c_int, [C.c_void_p, C.c_char_p, C.c_char_p, C.c_void_p, C.c_uint64, C.c_int]),
    ("gpudb_upload_column", C.c_int, [C.c_void_p, C.c_char_p, C.c_char_p, C.c_void_p, C.c_uint64, C.c_int]),
    ("gpudb_register_host_column", C.c_int, [C.c_void_p, C.c_char_p, C.c_char_p, C.c_void_p, C.c_uint64,
                                             C.c_int]),
    ("gpudb_colbin_inspect", C.c_int, [C.c_char_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint32),
                                       C.POINTER(ColbinColumn), C.c_uint32]),
    ("gpudb_colbin_load", C.c_int, [C.c_void_p, C.c_char_p, C.c_char_p, C.POINTER(ColbinLoadSpec), C.c_int]),
    ("gpudb_sql_to_spec", C.c_int, [C.c_char_p, C.c_char_p, C.c_size_t]),
    ("gpudb_register_rows", C.c_int, [C.c_void_p, C.c_char_p, C.c_uint64]),
    ("gpudb_register_buffer", C.c_int, [C.c_void_p, C.c_char_p, C.c_void_p, C.c_uint64, C.c_int]),
    ("gpudb_register_symbol", C.c_int, [C.c_void_p, C.c_char_p, C.c_uint64]),
    ("gpudb_get_symbol", C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(C.c_uint64)]),
    ("gpudb_register_scalar_i64", C.c_int, [C.c_void_p, C.c_char_p, C.c_longlong]),
    ("gpudb_register_scalar_f64", C.c_int, [C.c_void_p, C.c_char_p, C.c_double]),
    ("gpudb_execute", C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(PhaseDesc), C.c_int, C.c_int, C.c_int, C.c_int,
                                C.c_int, C.POINTER(Timing)]),
    ("gpudb_set_skip_zero_init", C.c_int, [C.c_void_p, C.c_int]),
    ("gpudb_set_use_graphs", C.c_int, [C.c_void_p, C.c_int]),
    ("gpudb_read_buffer", C.c_int, [C.c_void_p, C.c_char_p, C.c_void_p, C.c_uint64]),
    ("gpudb_buffer_ptr", C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(C.c_void_p), C.POINTER(C.c_uint64)]),
    ("gpudb_release_buffers", C.c_int, [C.c_void_p]),
    ("gpudb_host_alloc", C.c_void_p, [C.c_uint64]),
    ("gpudb_host_free", None, [C.c_void_p]),
    ("gpudb_distinct_count_noalloc", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_int32, C.c_int64,
                                               C.c_void_p, C.c_void_p]),
    # gpudb_engine.h: analyzed queries
    ("gpudb_aq_create", C.c_int, [C.POINTER(C.c_void_p)]),
    ("gpudb_aq_free", None, [C.c_void_p]),
    ("gpudb_aq_col", C.c_void_p, [C.c_void_p, C.c_char_p, C.c_char_p]),
    ("gpudb_aq_lit_int", C.c_void_p, [C.c_void_p, C.c_int64]),
    ("gpudb_aq_lit_decimal", C.c_void_p, [C.c_void_p, C.c_double]),
    ("gpudb_aq_lit_str", C.c_void_p, [C.c_void_p, C.c_char_p]),
    ("gpudb_aq_binary", C.c_void_p, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    ("gpudb_aq_cmp", C.c_void_p, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    ("gpudb_aq_between", C.c_void_p, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("gpudb_aq_in_list", C.c_void_p, [C.c_void_p, C.c_void_p, C.POINTER(C.c_void_p), C.c_int]),
    ("gpudb_aq_and", C.c_void_p, [C.c_void_p, C.POINTER(C.c_void_p), C.c_int]),
    ("gpudb_aq_or", C.c_void_p, [C.c_void_p, C.POINTER(C.c_void_p), C.c_int]),
    ("gpudb_aq_not", C.c_void_p, [C.c_void_p, C.c_void_p]),
    ("gpudb_aq_add_table", C.c_int, [C.c_void_p, C.c_char_p]),
    ("gpudb_aq_add_join", C.c_int, [C.c_void_p, C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p]),
    ("gpudb_aq_add_filter", C.c_int, [C.c_void_p, C.c_void_p]),
    ("gpudb_aq_add_target", C.c_int, [C.c_void_p, C.c_void_p, C.c_char_p]),
    ("gpudb_aq_add_agg", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_char_p]),
    ("gpudb_aq_add_group_by", C.c_int, [C.c_void_p, C.c_void_p]),
    ("gpudb_aq_add_order_by", C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    ("gpudb_aq_set_limit", C.c_int, [C.c_void_p, C.c_int]),
    ("gpudb_aq_lower_expr", C.c_int, [C.c_void_p, C.c_char_p, C.c_size_t, C.POINTER(C.c_int)]),
    ("gpudb_aq_lower_pred", C.c_int, [C.c_void_p, C.c_char_p, C.c_size_t]),
    ("gpudb_query_prepare_analyzed", C.c_int, [C.c_void_p, C.c_void_p, C.c_char_p, C.c_char_p,
                                               C.POINTER(C.c_void_p)]),
    # gpudb_engine.h
    ("gpudb_query_collect", C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_void_p)]),
    ("gpudb_query_prepare", C.c_int, [C.c_void_p, C.c_char_p, C.c_char_p, C.POINTER(C.c_void_p)]),
    ("gpudb_query_free", None, [C.c_void_p]),
    ("gpudb_query_source", C.c_size_t, [C.c_void_p, C.c_char_p, C.c_size_t]),
    ("gpudb_query_describe", C.c_size_t, [C.c_void_p, C.c_char_p, C.c_size_t]),
    ("gpudb_query_compile_log", C.c_size_t, [C.c_void_p, C.c_char_p, C.c_size_t]),
    ("gpudb_query_algorithmic_bytes", C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_longlong)]),
    ("gpudb_query_run", C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_void_p),
                                  C.POINTER(Timing)]),
    ("gpudb_query_run_streamed", C.c_int, [C.c_void_p, C.c_void_p, C.c_char_p, C.c_void_p, C.c_int, C.c_uint64,
                                           C.c_uint64, C.POINTER(C.c_void_p), C.POINTER(Timing)]),
    ("gpudb_query_enqueue", C.c_int, [C.c_void_p, C.c_void_p]),
    ("gpudb_ctx_sync", C.c_int, [C.c_void_p, C.POINTER(C.c_uint)]),
    ("gpudb_result_shape", C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_longlong)]),
    ("gpudb_result_column", C.c_int, [C.c_void_p, C.c_int, C.c_char_p, C.c_size_t, C.POINTER(C.c_int)]),
    ("gpudb_result_get_int", C.c_int, [C.c_void_p, C.c_longlong, C.c_int, C.POINTER(C.c_int64),
                                       C.POINTER(C.c_int64)]),
    ("gpudb_result_get_f64", C.c_int, [C.c_void_p, C.c_longlong, C.c_int, C.POINTER(C.c_double)]),
    ("gpudb_result_get_str", C.c_size_t, [C.c_void_p, C.c_longlong, C.c_int, C.c_char_p, C.c_size_t]),
    ("gpudb_result_export_i64", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_longlong]),
    ("gpudb_result_canonical", C.c_size_t, [C.c_void_p, C.c_int, C.c_char_p, C.c_size_t]),
    ("gpudb_result_free", None, [C.c_void_p]),
    ("gpudb_compare_canonical", C.c_int, [C.c_char_p, C.c_char_p, C.c_double, C.c_double, C.c_char_p,
                                          C.c_size_t]),
    ("gpudb_register_max_key", C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(C.c_longlong)]),
    ("gpudb_list_templates", C.c_size_t, [C.c_char_p, C.c_size_t]),
    ("gpudb_version", C.c_char_p, []),
    # gpudb_batch.h
    ("gpudb_sizer_create", C.c_int, [C.c_int, C.c_uint64, C.POINTER(C.c_void_p)]),
    ("gpudb_sizer_free", None, [C.c_void_p]),
    ("gpudb_sizer_param_count", C.c_int, []),
    ("gpudb_sizer_get_params", C.c_int, [C.c_void_p, C.c_void_p]),
    ("gpudb_sizer_set_params", C.c_int, [C.c_void_p, C.c_void_p]),
    ("gpudb_sizer_grads", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                    C.POINTER(C.c_float)]),
    ("gpudb_sizer_train", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_float,
                                    C.c_uint64, C.POINTER(C.c_float)]),
    ("gpudb_sizer_predict", C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    ("gpudb_column_minmax", C.c_int, [C.c_void_p, C.c_uint64, C.c_int, C.POINTER(C.c_int64),
                                      C.POINTER(C.c_int64), C.c_void_p]),
    ("gpudb_batch_create", C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    ("gpudb_batch_free", None, [C.c_void_p]),
    ("gpudb_batch_set_queries", C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    ("gpudb_batch_set_groups", C.c_int, [C.c_void_p, C.c_int, C.c_uint64]),
    ("gpudb_batch_set_agg_mode", C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    ("gpudb_batch_set_tuning", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int]),
    ("gpudb_batch_set_option", C.c_int, [C.c_void_p, C.c_char_p, C.c_longlong]),
    ("gpudb_batch_execute", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_double), C.c_void_p]),
    ("gpudb_batch_exact_stats", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_double)]),
    ("gpudb_batch_features", C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_double)]),
    ("gpudb_batch_result_scalar", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int64), C.POINTER(C.c_uint64),
                                            C.POINTER(C.c_int64)]),
    ("gpudb_batch_result_groups", C.c_int, [C.c_void_p, C.c_int, C.c_uint64, C.POINTER(C.c_uint64), C.c_void_p,
                                            C.c_void_p, C.c_void_p]),
    ("gpudb_batch_result_topk", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.POINTER(C.c_int)]),
    ("gpudb_batch_collect", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64),
                                      C.POINTER(C.c_double)]),
    ("gpudb_batch_last_launches", C.c_longlong, [C.c_void_p]),
    ("gpudb_batch_stage_ms", C.c_int, [C.c_void_p, C.c_void_p]),
]

_DATAGEN_SIGNATURES = [
    ("gpudb_gen_fact", C.c_int, [C.c_uint64, C.c_uint64, C.c_uint64] + [C.c_void_p] * 7 + [C.c_int]),
    ("gpudb_gen_dim", C.c_int, [C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64] + [C.c_void_p] * 3 + [C.c_int]),
    ("gpudb_gen_probe", C.c_int, [C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64] + [C.c_void_p] * 4 + [C.c_int]),
    ("gpudb_gen_order_day", C.c_int32, [C.c_uint64, C.c_int64]),
    ("gpudb_gen_zbuild", C.c_int, [C.c_uint64, C.c_uint64, C.c_uint64, C.c_void_p, C.c_void_p, C.c_int]),
    ("gpudb_gen_zprobe", C.c_int, [C.c_uint64, C.c_uint64, C.c_double, C.c_uint64, C.c_uint64, C.c_void_p,
                                   C.c_void_p, C.c_int]),
    ("gpudb_gen_zkey", C.c_int64, [C.c_uint64, C.c_uint64]),
    ("gpudb_gen_mix", C.c_int, [C.c_uint64, C.c_uint64, C.c_double, C.c_uint64, C.c_uint64, C.c_uint64]
     + [C.c_void_p] * 5 + [C.c_int]),
    ("gpudb_gen_mixdim", C.c_int, [C.c_uint64, C.c_uint64, C.c_uint64, C.c_void_p, C.c_void_p, C.c_int]),
    ("gpudb_gen_mix_device", C.c_int, [C.c_uint64, C.c_uint64, C.c_double, C.c_uint64, C.c_uint64, C.c_uint64]
     + [C.c_void_p] * 6),
    ("gpudb_gen_mixdim_device", C.c_int, [C.c_uint64, C.c_uint64, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("gpudb_datagen_last_error", C.c_char_p, []),
    ("gpudb_gen_snow_cust", C.c_int, [C.c_uint64, C.c_uint64, C.c_uint64, C.c_void_p, C.c_void_p, C.c_int]),
    ("gpudb_gen_snow_supp", C.c_int, [C.c_uint64, C.c_uint64, C.c_uint64, C.c_void_p, C.c_void_p, C.c_int]),
    ("gpudb_gen_snow_orders", C.c_int, [C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_int]),
    ("gpudb_gen_snow_lines", C.c_int, [C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64, C.c_void_p,
                                       C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
]

EXPORTED = [s[0] for s in _SIGNATURES]
DATAGEN_EXPORTED = [s[0] for s in _DATAGEN_SIGNATURES]

_lib = None
_datagen = None


class GpudbError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"gpudb {STATUS_NAMES.get(status, status)}: {message}")
        self.status = status
        self.message = message


def load() -> C.CDLL:
    """Load libgpudb.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: run gpudbmetalcodegen_b200.build_native.build() "
                           "(there is no fallback implementation)")
    lib = C.CDLL(str(LIB_PATH), mode=os.RTLD_NOW | getattr(os, "RTLD_GLOBAL", 0))
    for name, res, args in _SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def load_datagen() -> C.CDLL:
    """Load libgpudb_datagen.so, the seeded table generators (raises if it
    was not built). It maps no engine code."""
    global _datagen
    if _datagen is not None:
        return _datagen
    if not DATAGEN_PATH.exists():
        raise RuntimeError(f"{DATAGEN_PATH} is missing: run gpudbmetalcodegen_b200.build_native.build()")
    lib = C.CDLL(str(DATAGEN_PATH), mode=os.RTLD_NOW)
    for name, res, args in _DATAGEN_SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _datagen = lib
    return lib


def datagen_error() -> str:
    return (load_datagen().gpudb_datagen_last_error() or b"").decode(errors="replace")


def last_error(ctx) -> str:
    lib = load()
    n = lib.gpudb_last_error(ctx, None, 0)
    buf = C.create_string_buffer(n + 1)
    lib.gpudb_last_error(ctx, buf, n + 1)
    return buf.value.decode(errors="replace")


def check(status: int, ctx=None) -> None:
    if status != GPUDB_OK:
        raise GpudbError(status, last_error(ctx))


def get_string(fn, *args) -> str:
    n = fn(*args, None, 0)
    buf = C.create_string_buffer(n + 1)
    fn(*args, buf, n + 1)
    return buf.value.decode(errors="replace")
