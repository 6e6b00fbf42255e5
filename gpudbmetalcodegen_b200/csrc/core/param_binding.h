#pragma once
// ===================================================================
// CUDA parameter bindings, symbolic sizes and result schemas.
//
// Backend-neutral metadata shared by the code generator (which emits
// kernel signatures from it), the executor (which allocates, fills and
// binds buffers from it) and the result collector (which decodes output
// buffers from it).
//
// Follows the reference's binding model (codegen/core/metal_param_binding.h:
// MetalParamKind :29-35, MetalParamBinding :46-68, MetalSizeResolver :74-97,
// MetalResultSchema :103-144). Differences, all B200-driven:
//   * Every kernel argument is passed by value in an 8-byte slot (device
//     pointer or widened scalar) instead of a [[buffer(N)]] index, so the
//     executor can bind with cuLaunchKernel's void** array directly.
//   * 64-bit aggregates are native `unsigned long long` words; the
//     reference's lo/hi uint32 pair becomes a lo/hi pair of 64-bit words
//     that together hold an exact 128-bit sum (see gpudb_device.cuh,
//     gpudb_acc128_add).
//   * Every kernel also receives the device error word (ErrorWord) through
//     which overflow / timeout / bounds conditions reach the host.
// ===================================================================

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

namespace gpudb {

// Fibonacci-hashing multiplier (2^64 / golden ratio). The reference uses the
// 32-bit form 2654435769u (metal_param_binding.h:22) with the low bits of the
// product; the CUDA templates take the HIGH bits of the 64-bit product, which
// spreads both dense and random keys.
inline constexpr uint64_t kFibHashMul = 0x9E3779B97F4A7C15ull;

enum class CudaParamKind {
    TableData,       // const T* __restrict__        — a resident column
    TableSize,       // long long                    — row count of a table
    DeviceBuffer,    // T* (or const T*)             — executor-allocated scratch/output
    ConstantScalar,  // scalar by value              — registered with register_scalar_*
    ConstantData,    // const T* to uploaded host data
    ErrorWord,       // unsigned*                    — device error word, always last
    BufferLength,    // long long                    — element count of a named buffer
};

const char* paramKindName(CudaParamKind k);

inline std::string tableDataName(const std::string& table) { return "d_" + table; }
inline std::string tableSizeName(const std::string& table) { return "n_" + table; }

// Byte width of a CUDA C element type spelling used by the generator.
size_t cudaTypeBytes(const std::string& elementType);

struct CudaParamBinding {
    std::string name;          // argument name inside the kernel
    std::string cudaTypeDecl;  // full declaration without the name
    CudaParamKind kind = CudaParamKind::DeviceBuffer;
    std::string tableName;     // TableData / TableSize: owning table
    std::string elementType;   // "int", "long long", "unsigned char", ...
    std::string sizeExpr;      // element count, symbolic (resolved by CudaSizeResolver)
    bool zeroInit = false;     // memset before every run (fillByte)
    int fillByte = 0;          // 0x00 or 0xFF (sentinel -1 / empty hash key)
    bool readOnly = false;
    bool late = false;         // TableData read only for surviving rows (never staged)
    size_t hostCopyBytes = 0;  // ConstantData
    int argIndex = -1;         // position in the kernel's argument list

    size_t elemSizeBytes() const { return cudaTypeBytes(elementType); }
};

// ===================================================================
// Size resolver: symbol table + expression evaluator.
// Grammar (own recursive-descent parser, a superset of the reference's
// metal_param_binding.cpp:32-101 forms):
//   expr   := term (('+'|'-') term)*
//   term   := factor (('*'|'/'|'%') factor)*
//   factor := INT | SYMBOL | '(' expr ')' | FUNC '(' expr (',' expr)* ')'
//   FUNC   := pow2ceil | max | min | log2ceil
// ===================================================================
class CudaSizeResolver {
public:
    void registerSymbol(const std::string& name, uint64_t value) { symbols_[name] = value; }
    bool hasSymbol(const std::string& name) const { return symbols_.count(name) != 0; }
    uint64_t getSymbol(const std::string& name) const;
    uint64_t resolve(const std::string& expr) const;
    const std::unordered_map<std::string, uint64_t>& symbols() const { return symbols_; }

private:
    std::unordered_map<std::string, uint64_t> symbols_;
};

// ===================================================================
// Result schema: what a plan produces and how to decode it.
// ===================================================================
struct CudaResultSchema {
    enum Kind { NONE, MATERIALIZE, SCALAR_AGG, KEYED_AGG, HASH_AGG, TOPK, DIRECT_AGG };
    Kind kind = NONE;

    // MATERIALIZE (reference: counter + output columns)
    struct ColumnDesc {
        std::string displayName;
        std::string bufferName;
        std::string elementType;
    };
    std::vector<ColumnDesc> columns;
    std::string counterBuffer;

    // SCALAR_AGG: one row; each entry is a 1-word int64 or a 2-word split int128.
    struct ScalarAggEntry {
        std::string displayName;
        std::string buffer;
        bool isWide = false;   // 2 words (exact 128-bit)
        int scaleDown = 0;     // display divisor (exact value kept as integer)
    };
    std::vector<ScalarAggEntry> scalarAggs;

    // KEYED_AGG: numBuckets x valuesPerBucket u64 words.
    struct KeyedAggSlot {
        std::string name;
        int offset = 0;
        bool isWide = false;
        int scaleDown = 0;
    };
    // Derived FP64 column: num / den, evaluated once on the host.
    struct DerivedColumn {
        std::string name;
        std::string numerator;    // slot name
        std::string denominator;  // slot name
    };
    // Group-key label decoders: bucket -> key value for each group column.
    struct BucketKey {
        std::string name;
        int divisor = 1;          // key index = (bucket / divisor) % modulus
        int modulus = 1;
        std::vector<std::string> labels;
    };
    struct KeyedAggInfo {
        int numBuckets = 0;
        int valuesPerBucket = 0;
        std::string bufferName;
        std::vector<KeyedAggSlot> slots;
        std::vector<DerivedColumn> derived;
        std::vector<BucketKey> keys;
        std::string bucketName = "bucket";  // the bucket column's name when no keys decode it
    };
    KeyedAggInfo keyedAgg;

    // HASH_AGG: key array + per-slot aggregate arrays; empty key = ~0.
    struct HashAggInfo {
        std::string keyBuffer;
        std::string keyType;          // "long long" or "int"
        std::string capacitySymbol;   // size expression of the table
        std::string keyName = "key";
        struct Agg { std::string name; std::string buffer; };
        std::vector<Agg> aggs;
        std::vector<DerivedColumn> derived;
        bool sortByKey = true;
        // > 0: packed slots of this many u64 words in keyBuffer, word 0 =
        // ~key (0 empty), word 1 + j = aggregate j
        int packedStride = 0;
    };
    HashAggInfo hashAgg;

    // TOPK: k rows of (key, value) written by the top-k operator.
    struct TopKInfo {
        std::string keyBuffer;      // long long[k]
        std::string valueBuffer;    // long long[k]
        std::string countBuffer;    // unsigned long long[1]: rows written
        std::string keyName = "key";
        std::string valueName = "value";
        int k = 0;
        // further columns of the k rows, gathered on the device into
        // buffers of k elements (e.g. attributes of the top keys)
        struct Extra {
            std::string name, buffer, elementType;
        };
        std::vector<Extra> extra;
    };
    TopKInfo topk;

    // DIRECT_AGG: direct-address arrays of equal length (AtomicAgg /
    // AtomicCount outputs), one row (index, values...) per index where any
    // value is non-zero, in index order (reference: the host read-back of
    // direct-address aggregates, codegen_main.cpp:1105-1721).
    struct DirectAggInfo {
        std::string sizeExpr;
        std::string keyName = "bucket";
        struct Agg {
            std::string name, buffer;
        };
        std::vector<Agg> aggs;
    };
    DirectAggInfo directAgg;
};

}  // namespace gpudb
