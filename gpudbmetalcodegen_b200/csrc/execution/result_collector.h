#pragma once
// ===================================================================
// GenericResult + CudaResultCollector.
//
// Mirrors the reference's GenericResult / MetalResultCollector
// (codegen/execution/metal_result_collector.h:19-58): typed rows, a stable
// canonical CSV serialisation, and per-schema decoders (scalar agg, keyed
// agg skipping all-zero buckets — metal_result_collector.cpp:231-235 —,
// materialize). Differences: integers are exact (int64, or 128-bit for
// wide sums reconstructed from the two-word split), FP64 derived columns
// (averages) are computed once here, and hash-aggregate / top-k decoders
// are added. Buffers are read from device memory through a reader
// callback, so the collector itself is host-only code.
// ===================================================================
#include <cstdint>
#include <functional>
#include <string>
#include <variant>
#include <vector>

#include "../core/param_binding.h"

namespace gpudb {

using int128 = __int128;

struct GenericResult {
    struct Column {
        std::string name;
        std::string type;  // "int" (exact integer), "double", "string"
    };
    std::vector<Column> columns;
    using Value = std::variant<int128, double, std::string>;
    using Row = std::vector<Value>;
    std::vector<Row> rows;

    // Reference format: header line, CSV rows, doubles as %.4f.
    std::string toCanonical() const;
    // Full-precision variant used for exact parity (%.17g doubles).
    std::string toExact() const;
    void print(int limit = -1) const;
    bool empty() const { return rows.empty(); }
    size_t numRows() const { return rows.size(); }
    int columnIndex(const std::string& name) const;
};

std::string int128ToString(int128 v);

// Compare two canonical CSV blobs: columns matched by header name, row
// counts must agree, numbers within absTol + relTol*max(|a|,|b|), strings
// exact (semantics of the reference's --check, codegen_main.cpp:47-188).
// Returns "" on match, else a one-line reason.
std::string compareCanonical(const std::string& got, const std::string& expected, double absTol, double relTol);

// Reads `bytes` of buffer `name` into `dst`; returns false if absent.
using BufferReader = std::function<bool(const std::string& name, void* dst, size_t bytes)>;
// Resolves a size expression (for hash-table capacities).
using SizeEval = std::function<uint64_t(const std::string& expr)>;

class CudaResultCollector {
public:
    static GenericResult collect(const CudaResultSchema& schema, const BufferReader& read, const SizeEval& size);

private:
    static GenericResult collectScalarAgg(const CudaResultSchema& s, const BufferReader& read);
    static GenericResult collectKeyedAgg(const CudaResultSchema& s, const BufferReader& read);
    static GenericResult collectHashAgg(const CudaResultSchema& s, const BufferReader& read, const SizeEval& size);
    static GenericResult collectTopK(const CudaResultSchema& s, const BufferReader& read);
    static GenericResult collectMaterialize(const CudaResultSchema& s, const BufferReader& read, const SizeEval& size);
    static GenericResult collectDirectAgg(const CudaResultSchema& s, const BufferReader& read, const SizeEval& size);
};

}  // namespace gpudb
