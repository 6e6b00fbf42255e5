#pragma once
// ===================================================================
// CUDA operators — composable producer/consumer code generation.
//
// Same operator API as the reference (codegen/operators/metal_operators.h:
// MetalOperator::produce(MetalCodegen&, ConsumerFn) :26-31): each operator's
// produce() registers its parameters, emits code around its child's
// produce() and wraps the consumer callback. Operators and their argument
// meanings follow the reference one for one (Scan, Selection, ComputeExpr,
// BitmapBuild/Probe/AntiProbe, ArrayStore/Lookup, TGReduce, KeyedAgg,
// AtomicAgg, AtomicCount, Materialize); the emitted text is CUDA for
// sm_100a. New operators the reference lacks: BufferScan, HashBuild,
// HashProbe, HashGroupBy (GPU open addressing with 64-bit CAS) and TopK.
//
// Expressions are CUDA C++ strings over the column names, indexed by the
// scan's index variable (default "i"), exactly like the reference's
// exprToMetal output (metal_plan_builder.cpp:64-117). `_row` always holds
// the global 64-bit row index.
// ===================================================================

#include <memory>
#include <string>
#include <vector>

#include "../core/cuda_codegen.h"

namespace gpudb {

class CudaOperator {
public:
    virtual ~CudaOperator() = default;
    virtual void produce(CudaCodegen& cg, ConsumerFn consume) = 0;
    virtual std::string describe() const = 0;
};

class CudaUnaryOperator : public CudaOperator {
protected:
    std::unique_ptr<CudaOperator> child_;

public:
    explicit CudaUnaryOperator(std::unique_ptr<CudaOperator> child) : child_(std::move(child)) {}
    std::string describeChain() const;
};

// How a scan moves column bytes from HBM to the row loop.
struct ScanConfig {
    enum Mode { Direct, TmaBulk };
    Mode mode = TmaBulk;
    int tileRows = 0;      // rows per TMA tile (multiple of 16); 0 = about 24 KB of staged columns
    int stages = 4;        // TMA ring depth (clamped to the shared-memory budget)
    int prefetchRows = 0;  // rows whose probe bitmap words are loaded ahead (0 = off)
    int vectorRows = 0;    // consecutive rows per consumer thread, loaded with wide shared loads (0/1 = off)
    int l2Prefetch = 0;    // tiles beyond the ring the producer prefetches into L2 (0 = off)
    // automatic tiles rounded down to whole rounds of the consumer threads:
    // for consumers whose per-row work (lookups, atomics) makes a stage wait
    // on its slowest warp; a pure streaming reduction keeps the fuller tile
    bool wholeRounds = false;
};

// ------------------------------------------------------------------
// Leaf: grid-stride / TMA-staged scan over a resident columnar table.
// Reference: MetalGridStrideScan (metal_operators.cpp:28-49).
// Direct mode emits the reference's grid-stride loop with 64-bit indices.
// TmaBulk mode runs a persistent tile loop: thread 0 streams each tile's
// columns into a shared-memory ring with cp.async.bulk (evict-first L2
// hint, CTA-local destination only) signalled by per-stage mbarriers; all threads
// consume rows from shared memory; rows of a partial last tile (and all
// rows when a column is not 16-byte aligned) take the direct loop.
// ------------------------------------------------------------------
class CudaGridStrideScan : public CudaOperator {
public:
    struct ColumnDesc {
        std::string paramName;
        std::string cudaType;
        bool late = false;  // read at consumption through its global pointer, never staged
    };
    CudaGridStrideScan(const std::string& table, const std::string& rowVar = "row",
                       const std::string& idxVar = "i");
    // `late` columns are only touched by rows that survive earlier
    // selections (late materialisation): the TMA ring does not stage them.
    void addColumn(const std::string& paramName, const std::string& cudaType, bool late = false);
    void setConfig(const ScanConfig& c) { cfg_ = c; }
    void produce(CudaCodegen& cg, ConsumerFn consume) override;
    std::string describe() const override;
    const std::string& tableName() const { return tableName_; }
    const std::vector<ColumnDesc>& columns() const { return columns_; }

private:
    void emitPrefetchedRows(CudaCodegen& cg, ConsumerFn consume, int pf, const std::string& tileRows);
    void emitVectorRows(CudaCodegen& cg, ConsumerFn consume, int pf, int tile, const std::vector<long long>& off);

public:

private:
    std::string tableName_, rowVar_, idxVar_;
    std::vector<ColumnDesc> columns_;
    ScanConfig cfg_;
};

// Leaf: grid-stride loop over executor buffers of `countExpr` elements
// (e.g. the slots of a hash table). Consumers register the buffers.
class CudaBufferScan : public CudaOperator {
public:
    CudaBufferScan(const std::string& countName, const std::string& countExpr, const std::string& idxVar = "i");
    void produce(CudaCodegen& cg, ConsumerFn consume) override;
    std::string describe() const override;

private:
    std::string countName_, countExpr_, idxVar_;
};

// Leaf: visits the slot indices listed in `listBuffer` (u32), as many as
// the device counter `countBuffer` (u64) holds when the kernel runs — the
// used slots of a hash table built with a slot list. `idxVar` is the slot.
class CudaSlotListScan : public CudaOperator {
public:
    CudaSlotListScan(const std::string& listBuffer, const std::string& countBuffer, const std::string& idxVar = "i");
    // Table columns the rows read at the listed positions (a gather: the
    // list holds row indices of `table`).
    void addGatherColumn(const std::string& paramName, const std::string& cudaType, const std::string& table);
    // A buffer written next to the list (same positions): its entry for
    // the current position is read into the local `varName`.
    void addListColumn(const std::string& bufferName, const std::string& cudaType, const std::string& varName);
    void produce(CudaCodegen& cg, ConsumerFn consume) override;
    std::string describe() const override;
    // For a parent that runs its own loop over the list: declares the
    // list, its counter, its length and the gathered columns, and returns
    // the expression of the number of listed entries.
    std::string declareList(CudaCodegen& cg) const;
    const std::string& listBuffer() const { return list_; }
    const std::string& indexVar() const { return idxVar_; }

private:
    std::string list_, count_, idxVar_;
    struct Gather {
        std::string name, type, table;
    };
    std::vector<Gather> gathers_;
    struct ListColumn {
        std::string buffer, type, var;
    };
    std::vector<ListColumn> listColumns_;
};

// Selection: if (predicate) consume(). Reference: metal_operators.cpp:63-69.
// With setBitmapOut, the predicate is also written out as a selection
// bitmap of the scanned table (bit r = row r passed), built per warp: the
// lanes that share a 32-row word (__match_any_sync on row >> 5) OR their
// bits together (__reduce_or_sync, i.e. a warp ballot when the lanes hold
// consecutive rows) and one lane sets the word with one atomicOr. A later
// phase reads it back with CudaSelectionScan.
class CudaSelection : public CudaUnaryOperator {
public:
    CudaSelection(std::unique_ptr<CudaOperator> child, const std::string& predicate);
    void setBitmapOut(const std::string& bitmapName, const std::string& rowsExpr) {
        bitmapOut_ = bitmapName;
        bitmapRows_ = rowsExpr;
    }
    void produce(CudaCodegen& cg, ConsumerFn consume) override;
    std::string describe() const override;

private:
    std::string predicate_;
    std::string bitmapOut_, bitmapRows_;
};

// Leaf: visits the rows of `table` whose bit is set in a selection bitmap
// written by an earlier phase (CudaSelection::setBitmapOut). Each thread
// takes whole 32-row words (grid-stride); zero words cost one load and no
// row. The columns registered with addColumn are read at the selected rows
// through their global pointers (a gather), so columns needed only by
// selected rows are never streamed.
class CudaSelectionScan : public CudaOperator {
public:
    CudaSelectionScan(const std::string& table, const std::string& bitmapName, const std::string& idxVar = "i");
    void addColumn(const std::string& paramName, const std::string& cudaType);
    void produce(CudaCodegen& cg, ConsumerFn consume) override;
    std::string describe() const override;

private:
    std::string table_, bitmap_, idxVar_;
    std::vector<std::pair<std::string, std::string>> columns_;
};

// A small phase after a top-k: for each of the (at most k) entries of the
// index buffer `indexBuffer` (long long, count in `countBuffer`), gathers
// source[index] of each registered direct-address array into an output
// buffer of k elements — e.g. the build-side attributes of the top keys,
// which the reference's host post-processing reads from its order maps
// (codegen_main.cpp:1211-1248). Indices outside a source raise
// GPUDB_ERR_BOUNDS.
class CudaIndexGather : public CudaOperator {
public:
    CudaIndexGather(const std::string& indexBuffer, const std::string& countBuffer, int k);
    void addColumn(const std::string& sourceArray, const std::string& type, const std::string& outBuffer,
                   const std::string& displayName);
    void produce(CudaCodegen& cg, ConsumerFn consume) override;
    std::string describe() const override;

private:
    std::string index_, count_;
    int k_;
    struct Col {
        std::string src, type, out, name;
    };
    std::vector<Col> cols_;
};

// ComputeExpr: T var = expr; consume(). Reference: metal_operators.cpp:86-91.
class CudaComputeExpr : public CudaUnaryOperator {
public:
    CudaComputeExpr(std::unique_ptr<CudaOperator> child, const std::string& varName, const std::string& varType,
                    const std::string& expression);
    void produce(CudaCodegen& cg, ConsumerFn consume) override;
    std::string describe() const override;

private:
    std::string varName_, varType_, expression_;
};

// Bitmap build / probe / anti-probe over 32-bit words.
// Reference: metal_operators.cpp:108-165. Optional counter of newly set
// bits gives the exact number of distinct build keys (sizing pass).
class CudaBitmapBuild : public CudaUnaryOperator {
public:
    CudaBitmapBuild(std::unique_ptr<CudaOperator> child, const std::string& bitmapName, const std::string& keyExpr,
                    const std::string& sizeExpr);
    void setDistinctCounter(const std::string& counterName) { counter_ = counterName; }
    void produce(CudaCodegen& cg, ConsumerFn consume) override;
    std::string describe() const override;

private:
    std::string bitmapName_, keyExpr_, sizeExpr_, counter_;
};

class CudaBitmapProbe : public CudaUnaryOperator {
public:
    CudaBitmapProbe(std::unique_ptr<CudaOperator> child, const std::string& bitmapName, const std::string& keyExpr,
                    bool anti = false);
    // Also count the bitmap's set bits (its distinct keys) into the u64
    // counter `counterName`: after the probe's rows, each thread popcounts
    // a grid-stride share of the words, one atomic per warp. Lets the build
    // set bits without reading them back.
    void setPopcountInto(const std::string& counterName) { popcount_ = counterName; }
    void produce(CudaCodegen& cg, ConsumerFn consume) override;
    std::string describe() const override;

private:
    std::string bitmapName_, keyExpr_;
    std::string popcount_;
    bool anti_;
};

class CudaAntiBitmapProbe : public CudaBitmapProbe {
public:
    CudaAntiBitmapProbe(std::unique_ptr<CudaOperator> child, const std::string& bitmapName,
                        const std::string& keyExpr)
        : CudaBitmapProbe(std::move(child), bitmapName, keyExpr, true) {}
};

// Direct-address maps. Reference: metal_operators.cpp:185-225 (0xFF fill =
// sentinel -1 for int maps).
class CudaArrayStore : public CudaUnaryOperator {
public:
    CudaArrayStore(std::unique_ptr<CudaOperator> child, const std::string& arrayName, const std::string& keyExpr,
                   const std::string& valueExpr, const std::string& valueType = "int",
                   const std::string& sizeExpr = "");
    // Every index of the array is stored by the phase: no -1 sentinel fill.
    void setDense(bool on) { dense_ = on; }
    void produce(CudaCodegen& cg, ConsumerFn consume) override;
    std::string describe() const override;

private:
    std::string arrayName_, keyExpr_, valueExpr_, valueType_, sizeExpr_;
    bool dense_ = false;
};

class CudaArrayLookup : public CudaUnaryOperator {
public:
    CudaArrayLookup(std::unique_ptr<CudaOperator> child, const std::string& arrayName, const std::string& keyExpr,
                    const std::string& resultVar, const std::string& resultType = "int", long long sentinel = -1);
    void produce(CudaCodegen& cg, ConsumerFn consume) override;
    std::string describe() const override;

private:
    std::string arrayName_, keyExpr_, resultVar_, resultType_;
    long long sentinel_;
};

// ------------------------------------------------------------------
// Scalar reduction. Reference: MetalTGReduce (metal_operators.cpp:258-346):
// per-thread local sums, SIMD + threadgroup reduce, one atomic per TG.
// Here: per-thread int64, warp shuffle + smem block reduce, then one
// global RED per accumulator per block ("wide" = exact 128-bit split
// pair, "long" = one 64-bit word).
// ------------------------------------------------------------------
class CudaTGReduce : public CudaUnaryOperator {
public:
    struct Accumulator {
        std::string name, buffer, valueExpr, type;  // type: "wide" | "long" | "umax"
    };
    CudaTGReduce(std::unique_ptr<CudaOperator> child, const std::string& outputPrefix);
    void addAccumulator(const std::string& name, const std::string& valueExpr, const std::string& type = "wide",
                        const std::string& buffer = "");
    void setResultAlias(const std::string& displayName, int scaleDown = 0);
    void produce(CudaCodegen& cg, ConsumerFn consume) override;
    std::string describe() const override;

private:
    std::string outputPrefix_;
    std::vector<Accumulator> accumulators_;
    struct ResultInfo {
        std::string displayName;
        int scaleDown = 0;
    };
    std::vector<ResultInfo> resultInfos_;
};

// ------------------------------------------------------------------
// Few-group keyed aggregation. Reference: MetalKeyedAgg
// (metal_operators.cpp:375-502): thread-local arrays + TG reduction when
// all aggregates are adds and buckets <= 64, else per-row atomics.
// Here three strategies, chosen by size:
//   registers : buckets*aggs <= 64 — per-thread register accumulators
//               updated branch-free (predicated on the bucket id), block
//               reduce, one RED per non-zero (bucket, agg) per block;
//   shared    : buckets*valuesPerBucket <= 16384 words — per-block smem
//               table with shared 64-bit atomics, flushed non-zero words;
//   global    : per-row global atomics (add / min / max).
// Output: numBuckets x valuesPerBucket u64 words; a "wide" aggregate
// occupies words offset and offset+1 (exact 128-bit split pair).
// ------------------------------------------------------------------
class CudaKeyedAgg : public CudaUnaryOperator {
public:
    struct Aggregate {
        std::string name;
        int offset = 0;
        std::string valueExpr;
        std::string atomicOp;  // add | min | max
        bool isWide = false;
        int scaleDown = 0;
    };
    // Registers: predicated update of every bucket's accumulators per row;
    // RegistersSwitch: a switch on the bucket, each row updates only its own;
    // SharedPrivate: the reference's thread-local arrays (metal_operators.cpp:
    // 402-405) kept in shared memory instead of registers — every thread owns
    // buckets x aggregates 64-bit slots, a row adds into its own bucket's
    // slots by address (no switch, no divergence, few registers), and the
    // block sums each slot over its threads at the end.
    enum class Strategy { Auto, Registers, Shared, Global, RegistersSwitch, SharedPrivate };
    CudaKeyedAgg(std::unique_ptr<CudaOperator> child, const std::string& outputArrayName,
                 const std::string& bucketExpr, int numBuckets, int valuesPerBucket,
                 const std::string& sizeExpr = "");
    void addAggregate(const std::string& name, int offset, const std::string& valueExpr,
                      const std::string& atomicOp = "add", bool isWide = false, int scaleDown = 0);
    void setStrategy(Strategy s) { strategy_ = s; }
    Strategy chosenStrategy() const;
    void produce(CudaCodegen& cg, ConsumerFn consume) override;
    std::string describe() const override;

private:
    std::string outputArrayName_, bucketExpr_;
    int numBuckets_, valuesPerBucket_;
    std::string sizeExpr_;
    std::vector<Aggregate> aggregates_;
    Strategy strategy_ = Strategy::Auto;
};

// ------------------------------------------------------------------
// Direct-address atomic aggregation. Reference: MetalAtomicAgg
// (metal_operators.cpp:525-533). Options for skew: warp aggregation of
// equal buckets (__match_any_sync + peer tree sum, one atomic per distinct
// bucket per warp) and a per-block shared-memory cache of hot buckets.
// ------------------------------------------------------------------
class CudaAtomicAgg : public CudaUnaryOperator {
public:
    CudaAtomicAgg(std::unique_ptr<CudaOperator> child, const std::string& arrayName, const std::string& bucketExpr,
                  const std::string& valueExpr, const std::string& sizeExpr = "",
                  const std::string& elemType = "unsigned long long");
    // Further arrays updated at the same bucket (share warp aggregation
    // and the shared-memory cache), e.g. a count beside a sum.
    void addAggregate(const std::string& arrayName, const std::string& valueExpr);
    void setWarpAggregate(bool on) { warpAgg_ = on; }
    // `probe` = shared slots tried before a row goes to the global array
    // (0 = 2). Once the cache is full every cold row pays that many, and
    // hot keys settle near their home slot while it fills: on the Zipf hash
    // join, 2 probes took 1.81 ms against 2.39 ms for 16.
    void setSharedCache(int log2Slots, int probe = 0) {
        smemLog2_ = log2Slots;
        smemProbe_ = probe > 0 ? probe : 2;
    }
    void setZeroInit(bool on) { zeroInit_ = on; }
    void produce(CudaCodegen& cg, ConsumerFn consume) override;
    std::string describe() const override;

private:
    std::string arrayName_, bucketExpr_, valueExpr_, sizeExpr_, elemType_;
    std::vector<std::pair<std::string, std::string>> extra_;
    bool warpAgg_ = false;
    int smemLog2_ = 0;
    int smemProbe_ = 2;
    bool zeroInit_ = true;
};

// Histogram. Reference: MetalAtomicCount (metal_operators.cpp:550-594):
// TG-local histogram when the static size is <= 256. Here <= 8192 bins go
// to a shared-memory histogram flushed non-zero bins.
class CudaAtomicCount : public CudaUnaryOperator {
public:
    CudaAtomicCount(std::unique_ptr<CudaOperator> child, const std::string& arrayName,
                    const std::string& bucketExpr, const std::string& sizeExpr = "");
    void produce(CudaCodegen& cg, ConsumerFn consume) override;
    std::string describe() const override;

private:
    std::string arrayName_, bucketExpr_, sizeExpr_;
};

// Materialize selected rows. Reference: MetalMaterialize
// (metal_operators.cpp:618-643, one atomic per row). Here positions are
// reserved per warp from a ballot of the selection (one atomic per warp);
// rows beyond the capacity raise GPUDB_ERR_CAPACITY and are dropped.
class CudaMaterialize : public CudaUnaryOperator {
public:
    struct Column {
        std::string arrayName, type, valueExpr, displayName;
    };
    CudaMaterialize(std::unique_ptr<CudaOperator> child, const std::string& counterName,
                    const std::string& capacityExpr);
    void addColumn(const std::string& arrayName, const std::string& type, const std::string& valueExpr,
                   const std::string& displayName = "");
    // An intermediate result read by a later phase, not the plan's output.
    // Its 4-byte columns (one or two) are gathered per CTA in shared memory
    // and appended with one atomic per CTA: rows keep no order.
    void setIntermediate(bool on) { intermediate_ = on; }
    void produce(CudaCodegen& cg, ConsumerFn consume) override;
    std::string describe() const override;

private:
    std::string counterName_, capacityExpr_;
    std::vector<Column> columns_;
    bool intermediate_ = false;
};

// ------------------------------------------------------------------
// GPU hash tables (new; the reference builds its tables on the host).
// ------------------------------------------------------------------
// Linear: a key array and one array per aggregate. Bucket8: 64-bit keys
// probed 8 slots (one 64-byte line) at a time. Packed (group-by tables with
// 64-bit keys only): key and aggregates share one slot of a power-of-two
// number of words, so a row touches one 32-byte sector, not one per array.
enum class HashLayout { Linear, Bucket8, Packed };

// Slot count / log2 of a hash table requested with `capacityExpr` slots:
// rounded up to a power of two, at least 16 (one bucket8 group twice).
std::string hashSlotsExpr(const std::string& capacityExpr);
std::string hashLog2Expr(const std::string& capacityExpr);

// Build: insert keyExpr (64-bit or 32-bit keys) and store payloads at the
// key's slot. Capacity is a power of two (sizeExpr rounded up).
class CudaHashBuild : public CudaUnaryOperator {
public:
    CudaHashBuild(std::unique_ptr<CudaOperator> child, const std::string& tableName, const std::string& keyExpr,
                  const std::string& keyType, const std::string& capacityExpr, HashLayout layout = HashLayout::Linear,
                  int maxProbe = 128);
    void addPayload(const std::string& column, const std::string& type, const std::string& valueExpr);
    void produce(CudaCodegen& cg, ConsumerFn consume) override;
    std::string describe() const override;

private:
    struct Payload {
        std::string column, type, valueExpr;
    };
    std::string table_, keyExpr_, keyType_, capExpr_;
    HashLayout layout_;
    int maxProbe_;
    std::vector<Payload> payloads_;
};

// Probe: long long slotVar = find(keyExpr); if (slotVar >= 0) consume().
class CudaHashProbe : public CudaUnaryOperator {
public:
    CudaHashProbe(std::unique_ptr<CudaOperator> child, const std::string& tableName, const std::string& keyExpr,
                  const std::string& keyType, const std::string& capacityExpr, const std::string& slotVar = "_slot",
                  HashLayout layout = HashLayout::Linear, int maxProbe = 128);
    void addPayloadRead(const std::string& column, const std::string& type);
    void produce(CudaCodegen& cg, ConsumerFn consume) override;
    std::string describe() const override;

private:
    std::string table_, keyExpr_, keyType_, capExpr_, slotVar_;
    HashLayout layout_;
    int maxProbe_;
    std::vector<std::pair<std::string, std::string>> payloadReads_;
};

// High-cardinality hash group-by with 64-bit sums / counts per group.
// Options: warp aggregation (match_any on the key) and a per-block
// shared-memory table (2^log2 slots) absorbing heavy hitters before the
// global table; the block flushes it at the end.
class CudaHashGroupBy : public CudaUnaryOperator {
public:
    CudaHashGroupBy(std::unique_ptr<CudaOperator> child, const std::string& tableName, const std::string& keyExpr,
                    const std::string& keyType, const std::string& capacityExpr,
                    HashLayout layout = HashLayout::Linear, int maxProbe = 128);
    void addAggregate(const std::string& name, const std::string& valueExpr);  // "1" = count
    void setWarpAggregate(bool on) { warpAgg_ = on; }
    // `probe` as for CudaAtomicAgg::setSharedCache (0 = 8)
    void setSharedPreAgg(int log2Slots, int probe = 0) {
        smemLog2_ = log2Slots;
        smemProbe_ = probe > 0 ? probe : 8;
    }
    // Record every slot when its group is created in <table>_slotlist
    // (count in <table>_nslots): later phases visit only used slots.
    void setSlotList(bool on) { slotList_ = on; }
    // Device-sized table: the buffers are allocated for `boundExpr` groups
    // (a host size expression) and not filled by the executor; the slot
    // count is computed in the kernel from `groupsExpr`, device code over
    // the u64 counter buffers `counters` that earlier phases produced. A
    // CudaHashInit phase with the same arguments must run first.
    void setDeviceCapacity(const std::string& groupsExpr, const std::string& boundExpr,
                           const std::vector<std::string>& counters);
    // A warm tier between the shared-memory table and the main table: a
    // global table of 2^log2Slots slots (small enough to stay in L2) that
    // keeps the first keys to reach it, `probe` probes each; keys it cannot
    // place go to the main table. A CudaHashWarmFlush phase must follow to
    // add the warm entries into the main table (64-bit keys, host-sized).
    void setWarmTier(int log2Slots, int probe = 4) {
        warmLog2_ = log2Slots;
        warmProbe_ = probe;
    }
    void produce(CudaCodegen& cg, ConsumerFn consume) override;
    std::string describe() const override;

private:
    struct Agg {
        std::string name, valueExpr;
    };
    std::string table_, keyExpr_, keyType_, capExpr_;
    HashLayout layout_;
    int maxProbe_;
    std::vector<Agg> aggs_;
    bool warpAgg_ = true;
    int smemLog2_ = 0;
    int smemProbe_ = 8;
    int warmLog2_ = 0, warmProbe_ = 4;
    bool slotList_ = false;
    std::string devGroups_, devBound_;
    std::vector<std::string> devCounters_;
};

// The warm tier's flush: every key the warm table of a CudaHashGroupBy
// holds is added into its main table (its own phase, after the group-by's).
class CudaHashWarmFlush : public CudaOperator {
public:
    CudaHashWarmFlush(const std::string& tableName, const std::string& capacityExpr, HashLayout layout, int maxProbe,
                      const std::vector<std::string>& aggNames, int warmLog2, bool slotList);
    void produce(CudaCodegen& cg, ConsumerFn consume) override;
    std::string describe() const override;

private:
    std::string table_, capExpr_;
    HashLayout layout_;
    int maxProbe_;
    std::vector<std::string> aggs_;
    int warmLog2_;
    bool slotList_;
};

// Initialises the slots a device-sized group-by table will use (keys
// empty, aggregates zero) from the same counters, so no host round trip
// sizes the table between the phases that count and the one that groups.
class CudaHashInit : public CudaOperator {
public:
    CudaHashInit(const std::string& tableName, const std::string& keyType, HashLayout layout,
                 const std::vector<std::string>& aggNames, const std::string& groupsExpr,
                 const std::string& boundExpr, const std::vector<std::string>& counters);
    void produce(CudaCodegen& cg, ConsumerFn consume) override;
    std::string describe() const override;

private:
    std::string table_, keyType_;
    HashLayout layout_;
    std::vector<std::string> aggs_;
    std::string groups_, bound_;
    std::vector<std::string> counters_;
};

// Top-k (value desc, key asc) of the consumed (key, value) pairs.
// Per-thread register lists, warp shuffle merge, block merge in smem,
// last-block-done merge of the per-block lists (one launch).
// Reference: host top-k in codegen_main.cpp:1211-1248.
class CudaTopK : public CudaUnaryOperator {
public:
    CudaTopK(std::unique_ptr<CudaOperator> child, const std::string& outPrefix, const std::string& keyExpr,
             const std::string& valueExpr, int k, int maxBlocks = 296);
    void produce(CudaCodegen& cg, ConsumerFn consume) override;
    std::string describe() const override;

private:
    void produceOverList(CudaCodegen& cg, const CudaSlotListScan& list, ConsumerFn consume);
    std::string out_, keyExpr_, valueExpr_;
    int k_, maxBlocks_;
};

// ------------------------------------------------------------------
// GPU sort of group rows for an ORDER BY without LIMIT (the reference
// sorts its group rows on the host, codegen_main.cpp:1105-1721): rows of
// three int64 columns (key, count, value) in dense arrays, ordered by value
// descending, then key ascending. A merge sort in phases:
//   Chunks : each block sorts 2048-row chunks in shared memory (bitonic);
//   Merge p: runs of 2048 << p rows merge pairwise (merge path: each block
//            finds its output tile's split of the two runs by binary
//            search, stages both ranges in shared memory, and every thread
//            merges its own span); a pass whose runs already cover all rows
//            returns at once, so a plan carries passes for its largest size;
//   Emit   : the sorted rows go to the output arrays, in order.
// Rows live in two ping-pong buffer sets <prefix>_{k,c,v}{0,1}; the row
// count is read on the device from `countBuffer`.
// ------------------------------------------------------------------
class CudaSortPass : public CudaOperator {
public:
    enum class Mode { Chunks, Merge, Emit };
    static constexpr int kChunk = 2048;
    CudaSortPass(Mode mode, const std::string& prefix, const std::string& countBuffer, const std::string& capacityExpr,
                 int pass = 0);
    // Chunks: the dense input arrays (key, count, value).
    void setInput(const std::string& keys, const std::string& counts, const std::string& values);
    // Emit: output column names.
    void setOutputNames(const std::string& key, const std::string& count, const std::string& value);
    void produce(CudaCodegen& cg, ConsumerFn consume) override;
    std::string describe() const override;

private:
    Mode mode_;
    std::string prefix_, count_, cap_;
    int pass_;
    std::string inK_, inC_, inV_;
    std::string outK_ = "key", outC_ = "count", outV_ = "value";
};

}  // namespace gpudb
