/*
 * gpudb_rt.h — C-ABI of the B200 execution runtime (libgpudb.so).
 *
 * Drop-in boundary for the reference engine's Metal runtime layer
 * (codegen/execution/runtime_compiler.{h,cpp} and
 *  codegen/execution/metal_generic_executor.{h,cpp}). Plain pointers and
 * sizes only; no C++ types or exceptions cross this boundary. Every
 * function returns GPUDB_OK (0) or a negative GPUDB_E_* status; the text
 * of the last error of a context is available from gpudb_last_error().
 *
 * Threading: one gpudb_ctx per host thread (a context is not thread-safe),
 * as the reference used one MTL::CommandQueue per executor. All work is
 * ordered on the context's CUDA stream; calls that return results
 * synchronise that stream.
 */
#ifndef GPUDB_RT_H
#define GPUDB_RT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes --------------------------------------------------- */
#define GPUDB_OK 0
#define GPUDB_E_INVALID (-1)   /* bad argument / unknown name              */
#define GPUDB_E_PLAN (-2)      /* plan / spec / codegen error              */
#define GPUDB_E_ALLOC (-3)     /* device or host allocation failed         */
#define GPUDB_E_LAUNCH (-4)    /* launch configuration / launch failed     */
#define GPUDB_E_COMPILE (-5)   /* NVRTC compilation failed                 */
#define GPUDB_E_CUDA (-6)      /* CUDA runtime / driver error              */
#define GPUDB_E_DEVICE (-7)    /* kernel reported a device error word      */
#define GPUDB_E_NOGPU (-8)     /* no usable CUDA device                    */

/* Device error word bits (gpudb_timing.device_error). */
#define GPUDB_DEVERR_HASH_OVERFLOW 0x1u
#define GPUDB_DEVERR_WAIT_TIMEOUT 0x2u
#define GPUDB_DEVERR_BOUNDS 0x4u
#define GPUDB_DEVERR_SENTINEL_KEY 0x8u
#define GPUDB_DEVERR_CAPACITY 0x10u

typedef struct gpudb_ctx gpudb_ctx;
typedef struct gpudb_module gpudb_module;

/* Parameter kinds (reference: MetalParamKind, core/metal_param_binding.h:29-35). */
#define GPUDB_PARAM_TABLE_DATA 0
#define GPUDB_PARAM_TABLE_SIZE 1
#define GPUDB_PARAM_DEVICE_BUFFER 2
#define GPUDB_PARAM_CONSTANT_SCALAR 3
#define GPUDB_PARAM_CONSTANT_DATA 4
#define GPUDB_PARAM_ERROR_WORD 5
#define GPUDB_PARAM_BUFFER_LENGTH 6

/* One kernel argument (reference: MetalParamBinding, metal_param_binding.h:46-68).
 * Arguments are bound in array order, each passed in an 8-byte slot. */
typedef struct {
    const char* name;
    int kind;               /* GPUDB_PARAM_*                                   */
    const char* elem_type;  /* "int", "long long", "unsigned char", ...        */
    const char* table;      /* TABLE_*: owning table; BUFFER_LENGTH: buffer    */
    const char* size_expr;  /* element count (symbolic), or NULL               */
    int zero_init;          /* fill before every run with fill_byte            */
    int fill_byte;          /* 0x00 or 0xFF                                    */
    int read_only;
} gpudb_binding_desc;

/* One phase = one kernel (reference: MetalCodegen::PhaseInfo,
 * core/metal_codegen_base.h:136-145). */
typedef struct {
    const char* name;           /* kernel name in the module                */
    const char* scanned_table;  /* sizes the grid; NULL for buffer scans     */
    int block_size;             /* threads per block                         */
    int max_blocks;             /* 0 = no cap                                */
    int single_thread;
    int dynamic_smem_bytes;
    int tile_rows;              /* >0: one CTA per tile, persistent grid      */
    int rows_per_thread;
    const gpudb_binding_desc* bindings;
    int nbindings;
} gpudb_phase_desc;

/* Timing of one execute (reference: MetalExecutionResult, metal_generic_executor.h:23-44). */
#define GPUDB_MAX_PHASES 32
typedef struct {
    double total_ms;                      /* kernel time of one iteration      */
    int nphases;
    double phase_ms[GPUDB_MAX_PHASES];
    int phase_grid[GPUDB_MAX_PHASES];
    int phase_block[GPUDB_MAX_PHASES];
    unsigned device_error;                /* OR of GPUDB_DEVERR_* bits         */
    long long launches;                   /* kernels launched per iteration    */
    double alloc_ms, plan_ms, codegen_ms, compile_ms, collect_ms;
} gpudb_timing;

/* ---- context (reference: MetalGenericExecutor ctor/dtor,
 *      metal_generic_executor.h:48-57, .cpp:13-21) ---------------------- */
int gpudb_create(int device, gpudb_ctx** out);
void gpudb_destroy(gpudb_ctx* ctx);
/* Copies the context's last error text; returns its full length. A NULL
 * ctx reports the last error of gpudb_create on this thread. */
size_t gpudb_last_error(gpudb_ctx* ctx, char* buf, size_t cap);
/* The context's CUDA stream (cudaStream_t), for callers that order their
 * own work (events, copies) with the engine's. */
void* gpudb_stream(gpudb_ctx* ctx);
int gpudb_device_info(gpudb_ctx* ctx, int* num_sms, int* cc_major, int* cc_minor);
int gpudb_synchronize(gpudb_ctx* ctx);

/* ---- compile (reference: RuntimeCompiler::compile / getPipeline,
 *      execution/runtime_compiler.h:15-18, .cpp:20-68) ----------------- */
/* Compiles CUDA source for sm_100a with NVRTC (cached by source hash) and
 * loads it, resolving `kernels`. Works without a GPU only for
 * gpudb_compile_check. */
int gpudb_compile(gpudb_ctx* ctx, const char* src, const char* const* kernels, int nkernels, gpudb_module** out);
void gpudb_module_free(gpudb_module* m);
/* Compile-only (no GPU needed): returns GPUDB_OK or GPUDB_E_COMPILE, copying
 * the NVRTC log (ptxas resource lines included) into log. */
int gpudb_compile_check(const char* src, char* log, size_t cap, double* compile_ms);
/* Reference: RuntimeCompiler::setFastMathEnabled (runtime_compiler.h:27). */
void gpudb_set_fast_math(int on);
void gpudb_set_kernel_cache_dir(const char* dir);

/* ---- registration (reference: MetalGenericExecutor::register*,
 *      metal_generic_executor.h:60-78) ---------------------------------- */
/* registerTableBuffer: a resident device column of `rows` elements. */
int gpudb_register_column(gpudb_ctx* ctx, const char* table, const char* column, const void* dptr, uint64_t rows,
                          int elem_bytes);
/* Copy a host column into a context-owned device buffer and register it
 * (the reference's zero-copy newBuffer(ptr) becomes one H2D upload into
 * resident HBM; host memory from gpudb_host_alloc is pinned). */
int gpudb_upload_column(gpudb_ctx* ctx, const char* table, const char* column, const void* host, uint64_t rows,
                        int elem_bytes);
/* The reference's zero-copy column (newBuffer(ptr), the kernel reads host
 * memory in place) for columns a plan reads late: `host` must be pinned
 * (gpudb_host_alloc); kernels read it over the host link only for rows that
 * survive the earlier selections. Executing a plan that reads it for every
 * row fails (status < 0, message in gpudb_last_error) instead of streaming it. */
int gpudb_register_host_column(gpudb_ctx* ctx, const char* table, const char* column, const void* host,
                               uint64_t rows, int elem_bytes);

/* ---- .colbin v2 ingest (reference: colbin::loadColumnsFromBinary,
 *      src/infra.h:583-670; format src/infra.h:512-560) ----------------
 * A .colbin file: 48-byte header (magic "TPCHCB01", version 2, column
 * count, row count), 32-byte column descriptors, 16 KiB-aligned payloads.
 * The file is memory-mapped and checked the way the reference checks it
 * (magic, version, directory and payloads inside the file, payload bytes =
 * rows x type width). */
typedef struct gpudb_colbin_column {
    int32_t column_index; /* source .tbl field index */
    uint8_t dtype;        /* 0 int32, 1 float32, 2 date YYYYMMDD (int32), 3 char, 4 fixed-width chars */
    uint16_t fixed_width; /* bytes per value of dtype 4 */
    uint64_t offset;      /* payload offset in the file */
    uint64_t size_bytes;
} gpudb_colbin_column;
/* Header and column directory of a .colbin file; no GPU needed. Up to
 * `cap` descriptors are copied; *ncols receives the file's count. */
int gpudb_colbin_inspect(const char* path, uint64_t* rows, uint32_t* ncols, gpudb_colbin_column* cols, uint32_t cap);

#define GPUDB_COLBIN_AS_IS 0   /* int32 / date / char stored at the engine column's width */
#define GPUDB_COLBIN_WIDEN 1   /* int32 or date -> int64 */
#define GPUDB_COLBIN_DECIMAL 2 /* float32 -> int64 round(x * scale): the engine's exact fixed point */
#define GPUDB_COLBIN_DAYS 3    /* date YYYYMMDD -> int32 days since 1992-01-01 */
typedef struct gpudb_colbin_load_spec {
    int32_t column_index; /* source field index in the file */
    const char* column;   /* engine column of `table` it becomes */
    int32_t transform;    /* GPUDB_COLBIN_* */
    int32_t scale;        /* GPUDB_COLBIN_DECIMAL: e.g. 100 for cents */
} gpudb_colbin_load_spec;
/* Upload the listed columns of a .colbin file into resident HBM as
 * `table`'s columns (as gpudb_upload_column does), converting each to the
 * engine column's type. The engine column's width must match the
 * transform's result. Returns once the copies are complete. */
int gpudb_colbin_load(gpudb_ctx* ctx, const char* path, const char* table, const gpudb_colbin_load_spec* specs,
                      int n);
/* registerTableRowCount. */
int gpudb_register_rows(gpudb_ctx* ctx, const char* table, uint64_t rows);
/* registerAllocatedBuffer: caller-owned device buffer (not freed). */
int gpudb_register_buffer(gpudb_ctx* ctx, const char* name, void* dptr, uint64_t bytes, int elem_bytes);
/* registerSymbol / tryGetSymbol. */
int gpudb_register_symbol(gpudb_ctx* ctx, const char* name, uint64_t value);
int gpudb_get_symbol(gpudb_ctx* ctx, const char* name, uint64_t* value);
/* registerScalarInt / registerScalarFloat. */
int gpudb_register_scalar_i64(gpudb_ctx* ctx, const char* name, long long value);
int gpudb_register_scalar_f64(gpudb_ctx* ctx, const char* name, double value);

/* ---- execute (reference: MetalGenericExecutor::execute,
 *      metal_generic_executor.h:81-99, .cpp:289-399) ------------------- */
int gpudb_execute(gpudb_ctx* ctx, gpudb_module* m, const gpudb_phase_desc* phases, int nphases, int first, int last,
                  int warmup, int measured, gpudb_timing* timing);
/* setSkipZeroInit (metal_generic_executor.h:105). */
int gpudb_set_skip_zero_init(gpudb_ctx* ctx, int skip);
/* Replay whole iterations as CUDA graphs. A launch sequence (kernels,
 * grids, arguments, fills) is captured when it recurs: on its second run,
 * or at once when one call repeats it (warmup + measured > 1); its first
 * single run is eager. A context keeps 512 graphs, the oldest dropped
 * first. */
int gpudb_set_use_graphs(gpudb_ctx* ctx, int on);

/* ---- results / lifetime (reference: getAllocatedBuffer /
 *      releaseAllocatedBuffers, metal_generic_executor.h:110-119) ------ */
int gpudb_read_buffer(gpudb_ctx* ctx, const char* name, void* host, uint64_t bytes);
int gpudb_buffer_ptr(gpudb_ctx* ctx, const char* name, void** dptr, uint64_t* bytes);
int gpudb_release_buffers(gpudb_ctx* ctx);

/* ---- pinned host memory for uploads / readback ----------------------- */
void* gpudb_host_alloc(uint64_t bytes);
void gpudb_host_free(void* p);

/* ---- allocation-free distinct count ---------------------------------- */
/* No counterpart in the reference: an entry point for callers that cannot
 * allocate device memory on the call path (hosts whose own allocator owns
 * all device memory, strict memory budgets). Counts the distinct values
 * of key[i] % card over rows with filter[i] < thr and writes the count to
 * *out_count (device pointer). For non-negative keys that is the result of
 * the "distinct" pipeline; a negative key is skipped here, where that
 * pipeline reports a bounds error instead. All work runs
 * on `stream` (a cudaStream_t; NULL = legacy default stream). Inputs and
 * the output are the caller's device buffers; the scratch bitmap is a
 * static device array sized for card <= 2^22 (512 KiB, held by every GPU
 * that loads the library). card outside [1, 2^22] -> GPUDB_E_INVALID.
 * n = 0 writes 0. Calls share the scratch: calls that overlap on the GPU
 * race. The first call on a device resolves the scratch address; that
 * address is kept for the life of the
 * process, so a device reset (cudaDeviceReset, or destroying the primary
 * context) invalidates this entry point for that device. Asynchronous:
 * read *out_count after the stream has completed. */
int gpudb_distinct_count_noalloc(const int32_t* key, const int32_t* filter, uint64_t n, int32_t thr, int64_t card,
                                 uint64_t* out_count, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GPUDB_RT_H */
