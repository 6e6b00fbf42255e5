#include "cuda_operators.h"

#include <sstream>
#include <stdexcept>

namespace gpudb {

namespace {

std::string S(long long v) { return std::to_string(v); }

// Key type -> (unsigned storage type, insert fn, find fn, empty literal).
struct KeyOps {
    std::string store, ins, find, empty, cast;
};
KeyOps keyOps(const std::string& keyType, HashLayout layout, bool packedOk = false) {
    if (layout == HashLayout::Packed) {
        if (!packedOk) throw std::runtime_error("the packed hash layout is for group-by tables only");
        if (keyType != "long long" && keyType != "unsigned long long")
            throw std::runtime_error("the packed hash layout needs 64-bit keys");
        return {"unsigned long long", "gpudb_htp_insert64", "", "0ull", "(unsigned long long)"};
    }
    if (keyType == "int" || keyType == "unsigned") {
        if (layout == HashLayout::Bucket8)
            throw std::runtime_error("Bucket8 hash layout needs 64-bit keys");
        return {"unsigned", "gpudb_ht_insert32", "gpudb_ht_find32", "GPUDB_EMPTY32", "(unsigned)"};
    }
    if (keyType == "long long" || keyType == "unsigned long long") {
        if (layout == HashLayout::Bucket8)
            return {"unsigned long long", "gpudb_htb_insert64", "gpudb_htb_find64", "GPUDB_EMPTY64",
                    "(unsigned long long)"};
        return {"unsigned long long", "gpudb_ht_insert64", "gpudb_ht_find64", "GPUDB_EMPTY64",
                "(unsigned long long)"};
    }
    throw std::runtime_error("hash key type must be int or long long, got '" + keyType + "'");
}

// Bucket8 probes count buckets of 8 slots; keep the same slot budget.
int probeArg(HashLayout layout, int maxProbe) {
    return layout == HashLayout::Bucket8 ? (maxProbe + 7) / 8 : maxProbe;
}

}  // namespace

std::string hashSlotsExpr(const std::string& capacityExpr) { return "pow2ceil(max(" + capacityExpr + ", 16))"; }
std::string hashLog2Expr(const std::string& capacityExpr) { return "log2ceil(max(" + capacityExpr + ", 16))"; }

std::string CudaUnaryOperator::describeChain() const { return child_ ? child_->describe() : ""; }

// ===================================================================
// CudaGridStrideScan
// ===================================================================
CudaGridStrideScan::CudaGridStrideScan(const std::string& table, const std::string& rowVar,
                                       const std::string& idxVar)
    : tableName_(table), rowVar_(rowVar), idxVar_(idxVar) {}

void CudaGridStrideScan::addColumn(const std::string& paramName, const std::string& cudaType, bool late) {
    for (const auto& c : columns_)
        if (c.paramName == paramName) return;
    columns_.push_back({paramName, cudaType, late});
}

void CudaGridStrideScan::produce(CudaCodegen& cg, ConsumerFn consume) {
    cg.setPhaseScannedTable(tableName_);
    if (columns_.empty())
        throw std::runtime_error("CudaGridStrideScan(" + tableName_ + "): no columns registered; call addColumn()");
    for (const auto& c : columns_) cg.addColumnParam(c.paramName, c.cudaType, tableName_, c.late);
    cg.addTableSizeParam(tableName_);
    bool anyStaged = false;
    for (const auto& c : columns_) anyStaged |= !c.late;
    const std::string n = tableSizeName(tableName_);
    const std::string& i = idxVar_;

    if (cfg_.mode == ScanConfig::Direct || !anyStaged) {
        cg.addComment("grid-stride scan of " + tableName_ + " (direct coalesced loads)");
        cg.addBlock("for (long long " + i + " = tid; " + i + " < " + n + "; " + i + " += tpg)", [&]() {
            cg.addLine("const long long _row = " + i + "; (void)_row;");
            consume();
        });
        return;
    }

    // ---- TMA bulk staged tile loop ------------------------------------
    const int bs = cg.currentThreadgroupSize();
    int tile = cfg_.tileRows;
    if (tile <= 0) {
        // auto: about 24 KB of staged columns per stage, 1024..8192 rows
        long long rowBytes = 0;
        for (const auto& c : columns_)
            if (!c.late) rowBytes += (long long)cudaTypeBytes(c.cudaType);
        tile = 1024;
        while (tile < 8192 && (long long)tile * 2 * rowBytes <= 24 * 1024) tile *= 2;
        // ... rounded down, when the plan asks, to whole rounds of the
        // consumer threads (every warp but the producer), each taking one
        // row or one vector group per round: a tile with a partial last
        // round gives some warps one more round than the rest, and the stage
        // waits for the slowest (measured on B200: the join probe over
        // 2048-row tiles and 480 consumers, 152 us; over 1920 rows, 144 us;
        // a streaming Q6 reduction over 1024 rows, 30.3 us; over 896, 30.8 us)
        const int unit = (bs - 32) * (cfg_.vectorRows > 1 ? cfg_.vectorRows : 1);
        if (cfg_.wholeRounds && unit > 0 && unit <= tile) tile = tile / unit * unit;
    }
    int stages = cfg_.stages;
    if (tile <= 0 || tile % 16 != 0)
        throw std::runtime_error("CudaGridStrideScan: tileRows must be a positive multiple of 16");
    if (stages < 1 || stages > 8) throw std::runtime_error("CudaGridStrideScan: stages must be in [1,8]");
    std::vector<long long> off;
    long long stageBytes = 0, txBytes = 0;
    for (const auto& c : columns_) {
        const long long w = (long long)cudaTypeBytes(c.cudaType);
        off.push_back(stageBytes);
        if (c.late) continue;
        stageBytes += ((long long)tile * w + 127) / 128 * 128;
        txBytes += (long long)tile * w;
    }
    if (txBytes >= (1 << 20)) throw std::runtime_error("CudaGridStrideScan: tile too large for one mbarrier transaction");
    // Ring depth is clamped to what fits one CTA's shared memory (227 KB on
    // sm_100) next to the operators' own shared tables and reductions.
    constexpr long long kSmemBudget = 200 * 1024;
    const long long avail = kSmemBudget - 128 - cg.dynamicSmemBytes();
    if (stageBytes > avail)
        throw std::runtime_error("CudaGridStrideScan: one " + S(tile) + "-row tile (" + S(stageBytes) +
                                 " B) does not fit in shared memory; use fewer tile rows");
    if ((long long)stages * stageBytes > avail) stages = (int)(avail / stageBytes);
    if (bs < 64) throw std::runtime_error("CudaGridStrideScan: the TMA scan needs at least two warps per block");
    const int barOff = cg.allocDynamicSmem(128);
    const int ringOff = cg.allocDynamicSmem((int)(stageBytes * stages));
    cg.setPhaseTileRows(tile);

    const std::string SB = S(stageBytes), ST = S(stages), TL = S(tile);
    // Vector mode: V consecutive rows per consumer thread, every staged
    // column read with wide loads (its stage region is 128-byte aligned and
    // a group of V rows starts at a multiple of V * width).
    int vec = cfg_.vectorRows;
    if (vec > 1) {
        const bool pow2 = (vec & (vec - 1)) == 0 && vec <= 8;
        if (!pow2 || tile % vec != 0)
            throw std::runtime_error("CudaGridStrideScan: vector rows must be 2, 4 or 8 and divide the tile");
    }
    // The innermost bitmap probe above this scan, if no operator between
    // them defines names: its words are loaded for prefetchRows rows ahead.
    int pf = -1;
    if (cfg_.prefetchRows > 0) {
        const auto& hs = cg.scanHints();
        for (int h = (int)hs.size() - 1; h >= 0; --h) {
            if (hs[h].kind == CudaCodegen::ScanHint::Barrier) break;
            if (hs[h].kind == CudaCodegen::ScanHint::BitmapPrefetch) {
                pf = h;
                break;
            }
        }
    }
    cg.addComment("TMA-bulk staged scan of " + tableName_ + ": " + TL + "-row tiles, " + ST +
                  "-stage cp.async.bulk ring, " + S(txBytes) + " B per tile; warp 0 produces, the other warps consume");
    cg.addBlock("", [&]() {
        cg.addLine("unsigned long long* _sb_full = reinterpret_cast<unsigned long long*>(gpudb_smem + " + S(barOff) +
                   ");");
        cg.addLine("unsigned long long* _sb_empty = _sb_full + " + ST + ";");
        cg.addLine("unsigned char* _sb_ring = gpudb_smem + " + S(ringOff) + ";");
        cg.addLine("const long long _sb_n = " + n + ";");
        std::string alignExpr;
        for (size_t k = 0; k < columns_.size(); k++) {
            if (columns_[k].late) {
                // outer name for the consumers' tile-relative view of a late column
                cg.addLine("const " + columns_[k].cudaType + "* const _lt_" + columns_[k].paramName + " = " +
                           columns_[k].paramName + ";");
                continue;
            }
            alignExpr += (alignExpr.empty() ? "" : " | ") + std::string("(unsigned long long)") + columns_[k].paramName;
        }
        cg.addLine("const bool _sb_aligned = ((" + alignExpr + ") & 15ull) == 0ull;");
        cg.addLine("const long long _sb_ntiles = _sb_aligned ? (_sb_n / " + TL + "ll) : 0ll;");
        cg.addIf("threadIdx.x == 0", [&]() {
            cg.addBlock("for (int _s = 0; _s < " + ST + "; ++_s)", [&]() {
                cg.addLine("gpudb_mbar_init(_sb_full + _s, 1u);");
                cg.addLine("gpudb_mbar_init(_sb_empty + _s, (blockDim.x >> 5) - 1u);");
            });
            cg.addLine("gpudb_mbar_init_fence();");
        });
        cg.addLine("__syncthreads();");
        cg.addLine("bool _sb_ok = true;");
        cg.addBlock("if ((threadIdx.x >> 5) == 0)", [&]() {
            cg.addComment("producer: one lane streams tiles into the ring, refilling a stage once every consumer warp released it");
            cg.addBlock("if (threadIdx.x == 0)", [&]() {
                cg.addLine("const unsigned long long _sb_pol = gpudb_policy_evict_first();");
                cg.addLine("long long _sb_j = 0;");
                cg.addBlock("for (long long _sb_t = blockIdx.x; _sb_t < _sb_ntiles; _sb_t += gridDim.x, ++_sb_j)", [&]() {
                    cg.addLine("const int _s = (int)(_sb_j % " + ST + ");");
                    cg.addBlock("if (_sb_j >= " + ST + ")", [&]() {
                        cg.addLine("if (!gpudb_mbar_wait(_sb_empty + _s, (unsigned)(((_sb_j / " + ST +
                                   ") - 1) & 1), gpudb_err)) { _sb_ok = false; break; }");
                        cg.addLine("gpudb_fence_proxy_async();");
                    });
                    cg.addLine("unsigned char* _st = _sb_ring + (long long)_s * " + SB + "ll;");
                    cg.addLine("gpudb_mbar_expect_tx(_sb_full + _s, " + S(txBytes) + "u);");
                    for (size_t k = 0; k < columns_.size(); k++) {
                        if (columns_[k].late) continue;
                        const long long w = (long long)cudaTypeBytes(columns_[k].cudaType);
                        cg.addLine("gpudb_bulk_g2s_stream(_st + " + S(off[k]) + ", " + columns_[k].paramName + " + _sb_t * " +
                                   TL + "ll, " + S(tile * w) + "u, _sb_full + _s, _sb_pol);");
                    }
                    if (cfg_.l2Prefetch > 0) {
                        // keep the l2Prefetch rounds after the ring's in L2 (into L2 only)
                        cg.addLine("const long long _pf_t = _sb_t + (long long)" + S(stages + cfg_.l2Prefetch - 1) +
                                   " * gridDim.x;");
                        cg.addBlock("if (_pf_t < _sb_ntiles)", [&]() {
                            for (size_t k = 0; k < columns_.size(); k++) {
                                if (columns_[k].late) continue;
                                const long long w = (long long)cudaTypeBytes(columns_[k].cudaType);
                                cg.addLine("gpudb_bulk_prefetch_l2(" + columns_[k].paramName + " + _pf_t * " + TL + "ll, " +
                                           S(tile * w) + "u);");
                            }
                        });
                        cg.addBlock("if (_sb_j == 0)", [&]() {  // the first rounds beyond the ring
                            cg.addBlock("for (int _pr = 1; _pr < " + S(cfg_.l2Prefetch) + "; ++_pr)", [&]() {
                                cg.addLine("const long long _pq = _sb_t + (long long)(" + S(stages) +
                                           " + _pr - 1) * gridDim.x;");
                                cg.addBlock("if (_pq < _sb_ntiles)", [&]() {
                                    for (size_t k = 0; k < columns_.size(); k++) {
                                        if (columns_[k].late) continue;
                                        const long long w = (long long)cudaTypeBytes(columns_[k].cudaType);
                                        cg.addLine("gpudb_bulk_prefetch_l2(" + columns_[k].paramName + " + _pq * " + TL +
                                                   "ll, " + S(tile * w) + "u);");
                                    }
                                });
                            });
                        });
                    }
                });
                // Exit rule: the CTA must not exit while a bulk copy it issued
                // is still writing its shared memory. Normally the consumers
                // waited for every stage; after a timed-out wait (producer or
                // consumer side) the producer itself waits, again bounded, for
                // the last copy issued into each stage (tiles _sb_j - stages ..
                // _sb_j - 1) before the block may leave the ring.
                cg.addBlock("for (long long _dj = _sb_j > " + ST + " ? _sb_j - " + ST + " : 0; _dj < _sb_j; ++_dj)", [&]() {
                    cg.addLine("if (!gpudb_mbar_wait(_sb_full + (int)(_dj % " + ST + "), (unsigned)((_dj / " + ST +
                               ") & 1), gpudb_err)) { _sb_ok = false; break; }");
                });
            });
        }, " else {");
        cg.increaseIndent();
        cg.addComment("consumers: wait for a full stage, process its rows from shared memory, release it");
        cg.addLine("long long _sb_j = 0;");
        cg.addBlock("for (long long _sb_t = blockIdx.x; _sb_t < _sb_ntiles; _sb_t += gridDim.x, ++_sb_j)", [&]() {
            cg.addLine("const int _s = (int)(_sb_j % " + ST + ");");
            cg.addLine("if (!__all_sync(0xffffffffu, gpudb_mbar_wait(_sb_full + _s, (unsigned)((_sb_j / " + ST +
                       ") & 1), gpudb_err))) { _sb_ok = false; break; }");
            cg.addBlock("", [&]() {
                cg.addLine("const long long _sb_base = _sb_t * " + TL + "ll;");
                cg.addLine("const unsigned char* _sb_st = _sb_ring + (long long)_s * " + SB + "ll;");
                for (size_t k = 0; k < columns_.size(); k++) {
                    const auto& c = columns_[k];
                    if (c.late)
                        cg.addLine("const " + c.cudaType + "* " + c.paramName + " = _lt_" + c.paramName + " + _sb_base;");
                    else
                        cg.addLine("const " + c.cudaType + "* " + c.paramName + " = reinterpret_cast<const " + c.cudaType +
                                   "*>(_sb_st + " + S(off[k]) + ");");
                }
                if (vec > 1) {
                    emitVectorRows(cg, consume, pf, tile, off);  // releases the stage itself
                } else if (pf < 0) {
                    cg.addBlock("for (int " + i + " = (int)threadIdx.x - 32; " + i + " < " + TL + "; " + i +
                                    " += (int)blockDim.x - 32)",
                                [&]() {
                                    cg.addLine("const long long _row = _sb_base + " + i + "; (void)_row;");
                                    consume();
                                });
                } else {
                    emitPrefetchedRows(cg, consume, pf, TL);
                }
            });
            if (vec <= 1) {
                cg.addLine("__syncwarp();");
                cg.addLine("if ((threadIdx.x & 31u) == 0u) gpudb_mbar_arrive(_sb_empty + _s);");
            }
        });
        cg.decreaseIndent();
        cg.addLine("}");
        cg.addLine("_sb_ok = !__syncthreads_or(!_sb_ok);");
        cg.addComment("rows of the partial last tile (all rows if a column is not 16-byte aligned)");
        cg.addBlock("if (_sb_ok) for (long long " + i + " = _sb_ntiles * " + TL + "ll + tid; " + i + " < _sb_n; " + i +
                        " += tpg)",
                    [&]() {
                        cg.addLine("const long long _row = " + i + "; (void)_row;");
                        consume();
                    });
    });
}

// Consumer row loop of a staged tile with the bitmap words of hint `pf`
// loaded for prefetchRows rows before any of them is used: the loads are
// independent, so each thread keeps several L2 requests in flight instead
// of one per row.
void CudaGridStrideScan::emitPrefetchedRows(CudaCodegen& cg, ConsumerFn consume, int pf, const std::string& TL) {
    const int kPrefetchRows = cfg_.prefetchRows;
    const auto hint = cg.scanHints()[pf];
    std::string guard;
    for (size_t h = pf + 1; h < cg.scanHints().size(); ++h)
        if (cg.scanHints()[h].kind == CudaCodegen::ScanHint::Guard)
            guard += " && (" + cg.scanHints()[h].expr + ")";
    const std::string& i = idxVar_;
    const std::string U = S(kPrefetchRows);
    cg.addLine("const int _pf_step = (int)blockDim.x - 32;");
    cg.addBlock("for (int _pf_i0 = (int)threadIdx.x - 32; _pf_i0 < " + TL + "; _pf_i0 += " + U + " * _pf_step)", [&]() {
        cg.addLine("unsigned _pfw[" + U + "];");
        cg.addLine("#pragma unroll");
        cg.addBlock("for (int _pf_u = 0; _pf_u < " + U + "; ++_pf_u)", [&]() {
            cg.addLine("const int " + i + " = _pf_i0 + _pf_u * _pf_step;");
            cg.addLine("_pfw[_pf_u] = 0u;");
            cg.addBlock("if (" + i + " < " + TL + guard + ")", [&]() {
                cg.addLine("const long long _pf_k = (long long)(" + hint.expr + ");");
                cg.addLine("if ((unsigned long long)(_pf_k >> 5) < (unsigned long long)len_" + hint.bitmap + ") _pfw[_pf_u] = __ldg(" +
                           hint.bitmap + " + (_pf_k >> 5));");
            });
        });
        cg.addLine("#pragma unroll");
        cg.addBlock("for (int _pf_u = 0; _pf_u < " + U + "; ++_pf_u)", [&]() {
            cg.addLine("const int " + i + " = _pf_i0 + _pf_u * _pf_step;");
            cg.addBlock("if (" + i + " < " + TL + ")", [&]() {
                cg.addLine("const long long _row = _sb_base + " + i + "; (void)_row;");
                cg.setPrefetchVar(pf, "_pfw[_pf_u]");
                consume();
                cg.setPrefetchVar(pf, "");
            });
        });
    });
}

// Consumer row loop of a staged tile in groups of V consecutive rows. Each
// thread first copies all its groups' staged values from shared memory
// into registers (wide loads) and releases the stage, then runs the rows:
// the ring is refilled while rows with slow follow-up work (late-column
// reads, hash inserts) are still in flight, so one such row no longer
// holds the whole tile. Register arrays shadow the column names, so row
// expressions `col[i]` read registers; late columns are offset to the
// group. With a bitmap-probe hint and pf > 0, a group's V bitmap words are
// loaded together before any of its rows uses one.
void CudaGridStrideScan::emitVectorRows(CudaCodegen& cg, ConsumerFn consume, int pf, int tile,
                                        const std::vector<long long>& off) {
    const int V = cfg_.vectorRows;
    const int consumers = cg.currentThreadgroupSize() - 32;
    const int groups = tile / V;
    const int G = (groups + consumers - 1) / consumers;  // groups per consumer thread (compile time)
    const std::string& i = idxVar_;
    const std::string VS = S(V), GS = S(G);
    cg.addLine("const int _v_step = (int)blockDim.x - 32;");
    // load phase
    for (size_t k = 0; k < columns_.size(); k++) {
        const auto& c = columns_[k];
        if (!c.late) cg.addLine(c.cudaType + " _vr_" + c.paramName + "[" + GS + "][" + VS + "];");
    }
    cg.addLine("#pragma unroll");
    cg.addBlock("for (int _g = 0; _g < " + GS + "; ++_g)", [&]() {
        cg.addLine("const int _vg = (int)threadIdx.x - 32 + _g * _v_step;");
        cg.addBlock("if (_vg < " + S(groups) + ")", [&]() {
            for (size_t k = 0; k < columns_.size(); k++) {
                const auto& c = columns_[k];
                if (c.late) continue;
                const long long w = (long long)cudaTypeBytes(c.cudaType);
                cg.addLine("gpudb_vload<" + c.cudaType + ", " + VS + ">(_sb_st + " + S(off[k]) + " + (long long)_vg * " +
                           S(w * V) + ", _vr_" + c.paramName + "[_g]);");
            }
        });
    });
    cg.addComment("the staged values are in registers: release the stage now");
    cg.addLine("__syncwarp();");
    cg.addLine("if ((threadIdx.x & 31u) == 0u) gpudb_mbar_arrive(_sb_empty + _s);");
    // row phase
    cg.addLine("#pragma unroll");
    cg.addBlock("for (int _g = 0; _g < " + GS + "; ++_g)", [&]() {
        cg.addLine("const int _vg = (int)threadIdx.x - 32 + _g * _v_step;");
        cg.addBlock("if (_vg < " + S(groups) + ")", [&]() {
            cg.addLine("const long long _vbase = _sb_base + (long long)_vg * " + VS + ";");
            for (size_t k = 0; k < columns_.size(); k++) {
                const auto& c = columns_[k];
                if (c.late)
                    cg.addLine("const " + c.cudaType + "* " + c.paramName + " = _lt_" + c.paramName + " + _vbase;");
                else
                    cg.addLine("const " + c.cudaType + "* " + c.paramName + " = _vr_" + c.paramName + "[_g];");
            }
            std::string pfVar;
            if (pf >= 0 && cfg_.prefetchRows > 0) {
                const auto hint = cg.scanHints()[pf];
                std::string guard;
                for (size_t h = pf + 1; h < cg.scanHints().size(); ++h)
                    if (cg.scanHints()[h].kind == CudaCodegen::ScanHint::Guard)
                        guard += " && (" + cg.scanHints()[h].expr + ")";
                cg.addLine("unsigned _pfw[" + VS + "];");
                cg.addLine("#pragma unroll");
                cg.addBlock("for (int " + i + " = 0; " + i + " < " + VS + "; ++" + i + ")", [&]() {
                    cg.addLine("_pfw[" + i + "] = 0u;");
                    cg.addBlock("if (true" + guard + ")", [&]() {
                        cg.addLine("const long long _pf_k = (long long)(" + hint.expr + ");");
                        cg.addLine("if ((unsigned long long)(_pf_k >> 5) < (unsigned long long)len_" + hint.bitmap +
                                   ") _pfw[" + i + "] = __ldg(" + hint.bitmap + " + (_pf_k >> 5));");
                    });
                });
                pfVar = "_pfw[" + i + "]";
            }
            cg.addLine("#pragma unroll");
            cg.addBlock("for (int " + i + " = 0; " + i + " < " + VS + "; ++" + i + ")", [&]() {
                cg.addLine("const long long _row = _vbase + " + i + "; (void)_row;");
                if (!pfVar.empty()) cg.setPrefetchVar(pf, pfVar);
                consume();
                if (!pfVar.empty()) cg.setPrefetchVar(pf, "");
            });
        });
    });
}

std::string CudaGridStrideScan::describe() const {
    return std::string(cfg_.mode == ScanConfig::TmaBulk ? "TmaScan(" : "GridStrideScan(") + tableName_ + ")";
}

// ===================================================================
// CudaBufferScan
// ===================================================================
CudaBufferScan::CudaBufferScan(const std::string& countName, const std::string& countExpr, const std::string& idxVar)
    : countName_(countName), countExpr_(countExpr), idxVar_(idxVar) {}

void CudaBufferScan::produce(CudaCodegen& cg, ConsumerFn consume) {
    cg.addSizeScalarParam(countName_, "long long", countExpr_);
    const std::string& i = idxVar_;
    cg.addBlock("for (long long " + i + " = tid; " + i + " < " + countName_ + "; " + i + " += tpg)", [&]() {
        cg.addLine("const long long _row = " + i + "; (void)_row;");
        consume();
    });
}

std::string CudaBufferScan::describe() const { return "BufferScan(" + countName_ + " = " + countExpr_ + ")"; }

CudaSlotListScan::CudaSlotListScan(const std::string& listBuffer, const std::string& countBuffer,
                                   const std::string& idxVar)
    : list_(listBuffer), count_(countBuffer), idxVar_(idxVar) {}

void CudaSlotListScan::addGatherColumn(const std::string& paramName, const std::string& cudaType,
                                       const std::string& table) {
    gathers_.push_back({paramName, cudaType, table});
}

void CudaSlotListScan::addListColumn(const std::string& bufferName, const std::string& cudaType,
                                     const std::string& varName) {
    listColumns_.push_back({bufferName, cudaType, varName});
}

std::string CudaSlotListScan::declareList(CudaCodegen& cg) const {
    for (const auto& g : gathers_) cg.addColumnParam(g.name, g.type, g.table, true);
    for (const auto& c : listColumns_) cg.addReadBufferParam(c.buffer, c.type);
    cg.addReadBufferParam(list_, "unsigned");
    cg.addReadBufferParam(count_, "unsigned long long");
    cg.addBufferLengthParam("len_" + list_, list_);
    // the count comes from an earlier kernel: every thread reads it through
    // L1 rather than all warps queueing on its one L2 line
    return "(long long)min(__ldg(" + count_ + "), (unsigned long long)len_" + list_ + ")";
}

void CudaSlotListScan::produce(CudaCodegen& cg, ConsumerFn consume) {
    const std::string n = declareList(cg);
    const std::string& i = idxVar_;
    cg.addLine("const long long _sl_n = " + n + ";");
    cg.addBlock("for (long long _sl = tid; _sl < _sl_n; _sl += tpg)", [&]() {
        cg.addLine("const long long " + i + " = (long long)__ldcg(" + list_ + " + _sl);");
        cg.addLine("const long long _row = " + i + "; (void)_row;");
        for (const auto& c : listColumns_)
            cg.addLine("const " + c.type + " " + c.var + " = __ldcg(" + c.buffer + " + _sl);");
        consume();
    });
}

std::string CudaSlotListScan::describe() const { return "SlotListScan(" + list_ + "[0.." + count_ + "))"; }

// ===================================================================
// Selection / ComputeExpr
// ===================================================================
CudaSelection::CudaSelection(std::unique_ptr<CudaOperator> child, const std::string& predicate)
    : CudaUnaryOperator(std::move(child)), predicate_(predicate) {}

void CudaSelection::produce(CudaCodegen& cg, ConsumerFn consume) {
    if (!bitmapOut_.empty()) {
        // one bit per row of the scanned table, zero-filled before the run
        cg.addBufferParam(bitmapOut_, "unsigned", "(" + bitmapRows_ + ") / 32 + 1", true, 0);
        cg.addBufferLengthParam("len_" + bitmapOut_, bitmapOut_);
    }
    cg.pushScanHint({CudaCodegen::ScanHint::Guard, predicate_, ""});
    child_->produce(cg, [&]() {
        if (bitmapOut_.empty()) {
            cg.addIf(predicate_, [&]() { consume(); });
            return;
        }
        const std::string p = cg.fresh("_sp"), w = cg.fresh("_sw"), g = cg.fresh("_sg"), b = cg.fresh("_sb");
        cg.addLine("const bool " + p + " = (" + predicate_ + ");");
        cg.addBlock("", [&]() {
            cg.addComment("selection bitmap: lanes sharing a 32-row word OR their bits, one atomic per word");
            cg.addLine("const long long " + w + " = _row >> 5;");
            cg.addLine("const unsigned " + g + " = __match_any_sync(__activemask(), (unsigned long long)" + w + ");");
            cg.addLine("const unsigned " + b + " = __reduce_or_sync(" + g + ", " + p + " ? 1u << (unsigned)(_row & 31) : 0u);");
            cg.addBlock("if (" + b + " != 0u && (int)(threadIdx.x & 31u) == __ffs(" + g + ") - 1)", [&]() {
                cg.addLine("if ((unsigned long long)" + w + " < (unsigned long long)len_" + bitmapOut_ + ") atomicOr(" +
                           bitmapOut_ + " + " + w + ", " + b + "); else gpudb_set_error(gpudb_err, GPUDB_ERR_BOUNDS);");
            });
        });
        cg.addIf(p, [&]() { consume(); });
    });
    cg.popScanHint();
}

std::string CudaSelection::describe() const {
    return "Selection(" + predicate_ + (bitmapOut_.empty() ? "" : " -> bitmap " + bitmapOut_) + ")";
}

// ===================================================================
// CudaSelectionScan
// ===================================================================
CudaSelectionScan::CudaSelectionScan(const std::string& table, const std::string& bitmapName, const std::string& idxVar)
    : table_(table), bitmap_(bitmapName), idxVar_(idxVar) {}

void CudaSelectionScan::addColumn(const std::string& paramName, const std::string& cudaType) {
    columns_.push_back({paramName, cudaType});
}

void CudaSelectionScan::produce(CudaCodegen& cg, ConsumerFn consume) {
    for (const auto& c : columns_) cg.addColumnParam(c.first, c.second, table_, true);
    cg.addTableSizeParam(table_);
    cg.addReadBufferParam(bitmap_, "unsigned");
    cg.addBufferLengthParam("len_" + bitmap_, bitmap_);
    const std::string n = tableSizeName(table_);
    const std::string& i = idxVar_;
    cg.addComment("rows of " + table_ + " selected in " + bitmap_ + ": whole 32-row words per thread");
    cg.addLine("const long long _ss_words = min((long long)len_" + bitmap_ + ", (" + n + " + 31) / 32);");
    cg.addBlock("for (long long _ssw = tid; _ssw < _ss_words; _ssw += tpg)", [&]() {
        cg.addLine("unsigned _ssb = __ldcs(" + bitmap_ + " + _ssw);");
        cg.addBlock("while (_ssb)", [&]() {
            cg.addLine("const long long " + i + " = _ssw * 32 + (__ffs(_ssb) - 1);");
            cg.addLine("_ssb &= _ssb - 1u;");
            cg.addLine("if (" + i + " >= " + n + ") break;");
            cg.addLine("const long long _row = " + i + "; (void)_row;");
            consume();
        });
    });
}

std::string CudaSelectionScan::describe() const { return "SelectionScan(" + table_ + " where " + bitmap_ + ")"; }

// ===================================================================
// CudaIndexGather
// ===================================================================
CudaIndexGather::CudaIndexGather(const std::string& indexBuffer, const std::string& countBuffer, int k)
    : index_(indexBuffer), count_(countBuffer), k_(k) {}

void CudaIndexGather::addColumn(const std::string& sourceArray, const std::string& type, const std::string& outBuffer,
                                const std::string& displayName) {
    cols_.push_back({sourceArray, type, outBuffer, displayName});
}

void CudaIndexGather::produce(CudaCodegen& cg, ConsumerFn consume) {
    (void)consume;
    cg.addReadBufferParam(index_, "long long");
    cg.addReadBufferParam(count_, "unsigned long long");
    for (const auto& c : cols_) {
        cg.addReadBufferParam(c.src, c.type);
        cg.addBufferLengthParam("len_" + c.src, c.src);
        cg.addBufferParam(c.out, c.type, S(k_), true, 0);
    }
    cg.addLine("const long long _ig_n = min((long long)__ldcg(" + count_ + "), " + S(k_) + "ll);");
    cg.addBlock("for (long long _j = tid; _j < _ig_n; _j += tpg)", [&]() {
        cg.addLine("const long long _ix = __ldcg(" + index_ + " + _j);");
        for (const auto& c : cols_)
            cg.addLine("if ((unsigned long long)_ix < (unsigned long long)len_" + c.src + ") " + c.out + "[_j] = " + c.src +
                       "[_ix]; else gpudb_set_error(gpudb_err, GPUDB_ERR_BOUNDS);");
    });
    auto& rs = cg.resultSchema();
    for (const auto& c : cols_) rs.topk.extra.push_back({c.name, c.out, c.type});
}

std::string CudaIndexGather::describe() const {
    return "IndexGather(" + S((long long)cols_.size()) + " columns at " + index_ + "[0.." + count_ + "))";
}

CudaComputeExpr::CudaComputeExpr(std::unique_ptr<CudaOperator> child, const std::string& varName,
                                 const std::string& varType, const std::string& expression)
    : CudaUnaryOperator(std::move(child)), varName_(varName), varType_(varType), expression_(expression) {}

void CudaComputeExpr::produce(CudaCodegen& cg, ConsumerFn consume) {
    cg.pushScanHint({CudaCodegen::ScanHint::Barrier, "", ""});
    child_->produce(cg, [&]() {
        cg.addLine("const " + varType_ + " " + varName_ + " = " + expression_ + ";");
        consume();
    });
    cg.popScanHint();
}

std::string CudaComputeExpr::describe() const { return "ComputeExpr(" + varName_ + " = " + expression_ + ")"; }

// ===================================================================
// Bitmaps
// ===================================================================
CudaBitmapBuild::CudaBitmapBuild(std::unique_ptr<CudaOperator> child, const std::string& bitmapName,
                                 const std::string& keyExpr, const std::string& sizeExpr)
    : CudaUnaryOperator(std::move(child)), bitmapName_(bitmapName), keyExpr_(keyExpr), sizeExpr_(sizeExpr) {}

void CudaBitmapBuild::produce(CudaCodegen& cg, ConsumerFn consume) {
    cg.addBitmapWriteParam(bitmapName_, sizeExpr_);
    cg.addBufferLengthParam("len_" + bitmapName_, bitmapName_);
    if (!counter_.empty()) {
        cg.addAtomicBufferParam(counter_, "unsigned long long", "1");
        cg.addLine("unsigned long long _bm_fresh = 0ull;  // keys this thread was first to set");
    }
    child_->produce(cg, [&]() {
        cg.addLine("const long long _bk = (long long)(" + keyExpr_ + ");");
        cg.addBlock("if ((unsigned long long)(_bk >> 5) >= (unsigned long long)len_" + bitmapName_ + ")", [&]() {
            cg.addLine("gpudb_set_error(gpudb_err, GPUDB_ERR_BOUNDS);");
        }, " else {");
        cg.increaseIndent();
        if (counter_.empty()) {
            cg.addLine("gpudb_bitmap_set(" + bitmapName_ + ", _bk);");
        } else {
            cg.addLine("const unsigned _bbit = 1u << (unsigned)(_bk & 31);");
            // a bit already set costs a load, not an atomic round trip: bits
            // only go from 0 to 1 during the pass, so a stale 0 costs the
            // atomic and nothing else (a repeated key's word stays in cache)
            cg.addLine("if ((" + bitmapName_ + "[_bk >> 5] & _bbit) == 0u && (atomicOr(" + bitmapName_ +
                       " + (_bk >> 5), _bbit) & _bbit) == 0u) ++_bm_fresh;");
        }
        consume();
        cg.decreaseIndent();
        cg.addLine("}");
    });
    if (!counter_.empty()) {
        cg.addComment("distinct count: warp sum, one atomic per warp");
        cg.addLine("_bm_fresh = gpudb_warp_sum_u64(_bm_fresh);");
        cg.addLine("if ((threadIdx.x & 31u) == 0u && _bm_fresh) atomicAdd(" + counter_ + ", _bm_fresh);");
    }
}

std::string CudaBitmapBuild::describe() const { return "BitmapBuild(" + bitmapName_ + ", key=" + keyExpr_ + ")"; }

CudaBitmapProbe::CudaBitmapProbe(std::unique_ptr<CudaOperator> child, const std::string& bitmapName,
                                 const std::string& keyExpr, bool anti)
    : CudaUnaryOperator(std::move(child)), bitmapName_(bitmapName), keyExpr_(keyExpr), anti_(anti) {}

void CudaBitmapProbe::produce(CudaCodegen& cg, ConsumerFn consume) {
    cg.addBitmapReadParam(bitmapName_, "");
    cg.addBufferLengthParam("len_" + bitmapName_, bitmapName_);
    // a (non-anti) probe lets the TMA scan load its bitmap words ahead
    const int hint = anti_ ? -1 : cg.pushScanHint({CudaCodegen::ScanHint::BitmapPrefetch, keyExpr_, bitmapName_});
    child_->produce(cg, [&]() {
        const std::string k = cg.fresh("_pk");
        cg.addLine("const long long " + k + " = (long long)(" + keyExpr_ + ");");
        // Keys beyond the bitmap are simply absent (not an error on probe).
        const std::string inb = "(unsigned long long)(" + k + " >> 5) < (unsigned long long)len_" + bitmapName_;
        const std::string word = hint >= 0 ? cg.prefetchVar(hint) : std::string();
        const std::string t = word.empty() ? "gpudb_bitmap_test(" + bitmapName_ + ", " + k + ")"
                                           : "((" + word + " >> (unsigned)(" + k + " & 31)) & 1u)";
        cg.addIf(anti_ ? "!(" + inb + " && " + t + ")" : "(" + inb + ") && " + t, [&]() { consume(); });
    });
    if (hint >= 0) cg.popScanHint();
    if (!popcount_.empty()) {
        cg.addAtomicBufferParam(popcount_, "unsigned long long", "1");
        cg.addComment("distinct keys of " + bitmapName_ + ": popcount of a grid-stride share of its words, one atomic per warp");
        cg.addBlock("", [&]() {
            cg.addLine("unsigned long long _pc = 0ull;");
            cg.addLine("for (long long _w = tid; _w < len_" + bitmapName_ + "; _w += tpg) _pc += (unsigned long long)__popc(__ldg(" +
                       bitmapName_ + " + _w));");
            cg.addLine("_pc = gpudb_warp_sum_u64(_pc);");
            cg.addLine("if ((threadIdx.x & 31u) == 0u && _pc) atomicAdd(" + popcount_ + ", _pc);");
        });
    }
}

std::string CudaBitmapProbe::describe() const {
    return std::string(anti_ ? "AntiBitmapProbe(" : "BitmapProbe(") + bitmapName_ + ", key=" + keyExpr_ + ")";
}

// ===================================================================
// Direct-address maps
// ===================================================================
CudaArrayStore::CudaArrayStore(std::unique_ptr<CudaOperator> child, const std::string& arrayName,
                               const std::string& keyExpr, const std::string& valueExpr,
                               const std::string& valueType, const std::string& sizeExpr)
    : CudaUnaryOperator(std::move(child)),
      arrayName_(arrayName), keyExpr_(keyExpr), valueExpr_(valueExpr), valueType_(valueType), sizeExpr_(sizeExpr) {}

void CudaArrayStore::produce(CudaCodegen& cg, ConsumerFn consume) {
    cg.addBufferParam(arrayName_, valueType_, sizeExpr_, !dense_, 0xFF);
    cg.addBufferLengthParam("len_" + arrayName_, arrayName_);
    child_->produce(cg, [&]() {
        const std::string k = cg.fresh("_ak");
        cg.addLine("const long long " + k + " = (long long)(" + keyExpr_ + ");");
        cg.addBlock("if ((unsigned long long)" + k + " >= (unsigned long long)len_" + arrayName_ + ")", [&]() {
            cg.addLine("gpudb_set_error(gpudb_err, GPUDB_ERR_BOUNDS);");
        }, " else {");
        cg.increaseIndent();
        cg.addLine(arrayName_ + "[" + k + "] = (" + valueType_ + ")(" + valueExpr_ + ");");
        consume();
        cg.decreaseIndent();
        cg.addLine("}");
    });
}

std::string CudaArrayStore::describe() const {
    return "ArrayStore(" + arrayName_ + "[" + keyExpr_ + "] = " + valueExpr_ + ")";
}

CudaArrayLookup::CudaArrayLookup(std::unique_ptr<CudaOperator> child, const std::string& arrayName,
                                 const std::string& keyExpr, const std::string& resultVar,
                                 const std::string& resultType, long long sentinel)
    : CudaUnaryOperator(std::move(child)),
      arrayName_(arrayName), keyExpr_(keyExpr), resultVar_(resultVar), resultType_(resultType), sentinel_(sentinel) {}

void CudaArrayLookup::produce(CudaCodegen& cg, ConsumerFn consume) {
    cg.addReadBufferParam(arrayName_, resultType_);
    cg.addBufferLengthParam("len_" + arrayName_, arrayName_);
    cg.pushScanHint({CudaCodegen::ScanHint::Barrier, "", ""});
    struct Pop {
        CudaCodegen& c;
        ~Pop() { c.popScanHint(); }
    } pop{cg};
    child_->produce(cg, [&]() {
        const std::string k = cg.fresh("_lk");
        cg.addLine("const long long " + k + " = (long long)(" + keyExpr_ + ");");
        cg.addLine("const " + resultType_ + " " + resultVar_ + " = ((unsigned long long)" + k +
                   " < (unsigned long long)len_" + arrayName_ + ") ? " + arrayName_ + "[" + k + "] : (" + resultType_ +
                   ")(" + S(sentinel_) + "ll);");
        cg.addIf(resultVar_ + " != (" + resultType_ + ")(" + S(sentinel_) + "ll)", [&]() { consume(); });
    });
}

std::string CudaArrayLookup::describe() const {
    return "ArrayLookup(" + resultVar_ + " = " + arrayName_ + "[" + keyExpr_ + "])";
}

// ===================================================================
// CudaTGReduce
// ===================================================================
CudaTGReduce::CudaTGReduce(std::unique_ptr<CudaOperator> child, const std::string& outputPrefix)
    : CudaUnaryOperator(std::move(child)), outputPrefix_(outputPrefix) {}

void CudaTGReduce::addAccumulator(const std::string& name, const std::string& valueExpr, const std::string& type,
                                  const std::string& buffer) {
    if (type != "wide" && type != "long" && type != "umax")
        throw std::runtime_error("CudaTGReduce: type must be 'wide', 'long' or 'umax'");
    accumulators_.push_back({name, buffer.empty() ? outputPrefix_ + "_" + name : buffer, valueExpr, type});
}

void CudaTGReduce::setResultAlias(const std::string& displayName, int scaleDown) {
    resultInfos_.push_back({displayName, scaleDown});
}

void CudaTGReduce::produce(CudaCodegen& cg, ConsumerFn consume) {
    const int na = (int)accumulators_.size();
    if (na == 0) throw std::runtime_error("CudaTGReduce: no accumulators");
    for (const auto& a : accumulators_)
        cg.addAtomicBufferParam(a.buffer, "unsigned long long", a.type == "wide" ? "2" : "1");
    cg.addLine("unsigned long long _tr_acc[" + S(na) + "];");
    cg.addLine("#pragma unroll");
    cg.addLine("for (int _a = 0; _a < " + S(na) + "; ++_a) _tr_acc[_a] = 0ull;");
    child_->produce(cg, [&]() {
        for (int a = 0; a < na; a++) {
            const auto& acc = accumulators_[a];
            if (acc.type == "umax")
                cg.addLine("_tr_acc[" + S(a) + "] = max(_tr_acc[" + S(a) + "], (unsigned long long)(" + acc.valueExpr + "));");
            else
                cg.addLine("_tr_acc[" + S(a) + "] += (unsigned long long)(long long)(" + acc.valueExpr + ");");
        }
        consume();
    });
    cg.addComment("block reduction (warp shuffles + smem), one RED per accumulator per block");
    cg.addLine("__shared__ unsigned long long _tr_red[32 * " + S(na) + "];");
    cg.addLine("#pragma unroll");
    cg.addBlock("for (int _a = 0; _a < " + S(na) + "; ++_a)", [&]() {
        cg.addLine("unsigned long long _v = _tr_acc[_a];");
        cg.addBlock("switch (_a)", [&]() {
            for (int a = 0; a < na; a++)
                cg.addLine("case " + S(a) + ": _v = " +
                           (accumulators_[a].type == "umax" ? "gpudb_warp_max_u64(_v)" : "gpudb_warp_sum_u64(_v)") +
                           "; break;");
            cg.addLine("default: break;");
        });
        cg.addLine("if ((threadIdx.x & 31u) == 0u) _tr_red[(threadIdx.x >> 5) * " + S(na) + " + _a] = _v;");
    });
    cg.addLine("__syncthreads();");
    cg.addBlock("for (int _a = threadIdx.x; _a < " + S(na) + "; _a += blockDim.x)", [&]() {
        cg.addLine("unsigned long long _tot = 0ull;");
        cg.addBlock("switch (_a)", [&]() {
            for (int a = 0; a < na; a++) {
                const auto& acc = accumulators_[a];
                const std::string comb = acc.type == "umax" ? "_tot = max(_tot, _tr_red[_w * " + S(na) + " + _a]);"
                                                            : "_tot += _tr_red[_w * " + S(na) + " + _a];";
                std::string emit;
                if (acc.type == "umax") emit = "if (_tot) atomicMax(" + acc.buffer + ", _tot);";
                else if (acc.type == "wide") emit = "if (_tot) gpudb_acc128_add(" + acc.buffer + ", (long long)_tot);";
                else emit = "if (_tot) gpudb_acc64_add(" + acc.buffer + ", (long long)_tot);";
                cg.addLine("case " + S(a) + ": for (int _w = 0; _w < (int)(blockDim.x >> 5); ++_w) " + comb + " " + emit +
                           " break;");
            }
            cg.addLine("default: break;");
        });
    });
    for (size_t i = 0; i < accumulators_.size(); i++) {
        const auto& a = accumulators_[i];
        const std::string disp = i < resultInfos_.size() ? resultInfos_[i].displayName : a.name;
        const int sd = i < resultInfos_.size() ? resultInfos_[i].scaleDown : 0;
        cg.registerScalarAggColumn(disp, a.buffer, a.type == "wide", sd);
    }
}

std::string CudaTGReduce::describe() const {
    return "TGReduce(" + S((long long)accumulators_.size()) + " accumulators) <- " + describeChain();
}

// ===================================================================
// CudaKeyedAgg
// ===================================================================
CudaKeyedAgg::CudaKeyedAgg(std::unique_ptr<CudaOperator> child, const std::string& outputArrayName,
                           const std::string& bucketExpr, int numBuckets, int valuesPerBucket,
                           const std::string& sizeExpr)
    : CudaUnaryOperator(std::move(child)),
      outputArrayName_(outputArrayName), bucketExpr_(bucketExpr), numBuckets_(numBuckets),
      valuesPerBucket_(valuesPerBucket), sizeExpr_(sizeExpr) {}

void CudaKeyedAgg::addAggregate(const std::string& name, int offset, const std::string& valueExpr,
                                const std::string& atomicOp, bool isWide, int scaleDown) {
    if (atomicOp != "add" && atomicOp != "min" && atomicOp != "max")
        throw std::runtime_error("CudaKeyedAgg: atomicOp must be add/min/max");
    if (isWide && atomicOp != "add") throw std::runtime_error("CudaKeyedAgg: wide aggregates must be adds");
    if (offset < 0 || offset + (isWide ? 2 : 1) > valuesPerBucket_)
        throw std::runtime_error("CudaKeyedAgg: aggregate '" + name + "' does not fit in valuesPerBucket");
    aggregates_.push_back({name, offset, valueExpr, atomicOp, isWide, scaleDown});
}

CudaKeyedAgg::Strategy CudaKeyedAgg::chosenStrategy() const {
    bool allAdds = true;
    for (const auto& a : aggregates_)
        if (a.atomicOp != "add") allAdds = false;
    if (strategy_ != Strategy::Auto) {
        if (!allAdds && strategy_ != Strategy::Global)
            throw std::runtime_error("CudaKeyedAgg: min/max aggregates need the Global strategy");
        return strategy_;
    }
    if (!allAdds) return Strategy::Global;
    if (numBuckets_ * (int)aggregates_.size() <= 64 && numBuckets_ <= 16) return Strategy::RegistersSwitch;
    if ((long long)numBuckets_ * valuesPerBucket_ <= 16384) return Strategy::Shared;
    return Strategy::Global;
}

void CudaKeyedAgg::produce(CudaCodegen& cg, ConsumerFn consume) {
    const std::string sz = sizeExpr_.empty() ? S((long long)numBuckets_ * valuesPerBucket_) : sizeExpr_;
    cg.addAtomicBufferParam(outputArrayName_, "unsigned long long", sz);
    const int nb = numBuckets_, vpb = valuesPerBucket_, na = (int)aggregates_.size();
    const Strategy st = chosenStrategy();
    const std::string out = outputArrayName_;

    auto emitValues = [&]() {
        cg.addLine("const int _bucket = (int)(" + bucketExpr_ + ");");
        for (int j = 0; j < na; j++)
            cg.addLine("const long long _kv" + S(j) + " = (long long)(" + aggregates_[j].valueExpr + ");");
    };

    if (st == Strategy::Registers || st == Strategy::RegistersSwitch) {
        cg.addComment("keyed aggregation: per-thread register accumulators (" + S(nb) + " buckets x " + S(na) +
                      " aggregates), predicated on the bucket id");
        for (int j = 0; j < na; j++) {
            std::string init;
            for (int b = 0; b < nb; b++) init += (b ? ", " : "") + std::string("0ll");
            cg.addLine("long long _ka" + S(j) + "[" + S(nb) + "] = {" + init + "};");
        }
        child_->produce(cg, [&]() {
            emitValues();
            if (st == Strategy::RegistersSwitch) {
                // one path per bucket: a row pays only its own bucket's adds;
                // a warp executes the paths of the buckets its rows hit
                cg.addBlock("switch (_bucket)", [&]() {
                    for (int b = 0; b < nb; b++) {
                        std::string body = "case " + S(b) + ":";
                        for (int j = 0; j < na; j++) body += " _ka" + S(j) + "[" + S(b) + "] += _kv" + S(j) + ";";
                        cg.addLine(body + " break;");
                    }
                    cg.addLine("default: gpudb_set_error(gpudb_err, GPUDB_ERR_BOUNDS); break;");
                });
            } else {
                cg.addLine("#pragma unroll");
                cg.addBlock("for (int _b = 0; _b < " + S(nb) + "; ++_b)", [&]() {
                    cg.addLine("const bool _hit = (_bucket == _b);");
                    for (int j = 0; j < na; j++) cg.addLine("_ka" + S(j) + "[_b] += _hit ? _kv" + S(j) + " : 0ll;");
                });
            }
            consume();
        });
        const int nacc = nb * na;
        cg.addComment("block reduction, then one RED per non-zero (bucket, aggregate) per block");
        cg.addLine("long long _ka_all[" + S(nacc) + "];");
        cg.addLine("#pragma unroll");
        cg.addBlock("for (int _b = 0; _b < " + S(nb) + "; ++_b)", [&]() {
            for (int j = 0; j < na; j++) cg.addLine("_ka_all[_b * " + S(na) + " + " + S(j) + "] = _ka" + S(j) + "[_b];");
        });
        cg.addLine("__shared__ long long _ka_red[32 * " + S(nacc) + "];");
        cg.addLine("gpudb_block_partials<" + S(nacc) + ">(_ka_all, _ka_red);");
        cg.addBlock("for (int _a = threadIdx.x; _a < " + S(nacc) + "; _a += blockDim.x)", [&]() {
            cg.addLine("const long long _tot = gpudb_block_total(_ka_red, " + S(nacc) + ", _a);");
            cg.addLine("if (_tot == 0ll) continue;");
            cg.addLine("const int _b = _a / " + S(na) + ", _j = _a % " + S(na) + ";");
            cg.addBlock("switch (_j)", [&]() {
                for (int j = 0; j < na; j++) {
                    const auto& ag = aggregates_[j];
                    cg.addLine("case " + S(j) + ": " + (ag.isWide ? "gpudb_acc128_add(" : "gpudb_acc64_add(") + out +
                               " + _b * " + S(vpb) + " + " + S(ag.offset) + ", _tot); break;");
                }
                cg.addLine("default: break;");
            });
        });
    } else if (st == Strategy::SharedPrivate) {
        const int bs = cg.currentThreadgroupSize();
        const std::string BS = S(bs);
        // a count ("1") never exceeds a thread's rows: its slots are 32-bit
        // (one shared-memory wavefront per warp access instead of two)
        std::vector<bool> narrow(na, false);
        int nWide = 0, nNarrow = 0;
        std::vector<int> pos(na, 0);
        for (int j = 0; j < na; j++) {
            const std::string& v = aggregates_[j].valueExpr;
            narrow[j] = (v == "1" || v == "1ll" || v == "1u");
            pos[j] = narrow[j] ? nNarrow++ : nWide++;
        }
        const int accW = nb * nWide, accN = nb * nNarrow;
        // allocated before the scan below sizes its ring from what is left
        const int poff = cg.allocDynamicSmem(accW * bs * 8);
        const int noff = accN ? cg.allocDynamicSmem(accN * bs * 4) : 0;
        cg.addComment("keyed aggregation: thread-private accumulators in shared memory (" + S(nb) + " buckets x " +
                      S(na) + " aggregates per thread; slot (bucket * aggregates + aggregate) * " + BS +
                      " + thread, so a warp's lanes hit consecutive words; counts in 32-bit slots)");
        cg.addLine("if (blockDim.x > " + BS + "u) { gpudb_set_error(gpudb_err, GPUDB_ERR_BOUNDS); return; }");
        cg.addLine("unsigned long long* const _kp_all = reinterpret_cast<unsigned long long*>(gpudb_smem + " + S(poff) +
                   ");");
        cg.addLine("unsigned long long* const _kp = _kp_all + threadIdx.x;");
        cg.addLine("#pragma unroll");
        cg.addLine("for (int _a = 0; _a < " + S(accW) + "; ++_a) _kp[_a * " + BS + "] = 0ull;");
        if (accN) {
            cg.addLine("unsigned* const _kn_all = reinterpret_cast<unsigned*>(gpudb_smem + " + S(noff) + ");");
            cg.addLine("unsigned* const _kn = _kn_all + threadIdx.x;");
            cg.addLine("#pragma unroll");
            cg.addLine("for (int _a = 0; _a < " + S(accN) + "; ++_a) _kn[_a * " + BS + "] = 0u;");
        }
        child_->produce(cg, [&]() {
            emitValues();
            cg.addBlock("if ((unsigned)_bucket < " + S(nb) + "u)", [&]() {
                if (nWide) cg.addLine("unsigned long long* const _kq = _kp + _bucket * " + S(nWide * bs) + ";");
                if (nNarrow) cg.addLine("unsigned* const _kr = _kn + _bucket * " + S(nNarrow * bs) + ";");
                for (int j = 0; j < na; j++) {
                    if (narrow[j]) cg.addLine("_kr[" + S(pos[j] * bs) + "] += 1u;");
                    else cg.addLine("_kq[" + S(pos[j] * bs) + "] += (unsigned long long)_kv" + S(j) + ";");
                }
            }, " else { gpudb_set_error(gpudb_err, GPUDB_ERR_BOUNDS); }");
            consume();
        });
        cg.addComment("each warp sums whole slots over the block's threads, then one RED per non-zero slot");
        cg.addLine("__syncthreads();");
        cg.addBlock("for (int _a = (int)(threadIdx.x >> 5); _a < " + S(nb * na) + "; _a += (int)(blockDim.x >> 5))", [&]() {
            cg.addLine("const int _b = _a / " + S(na) + ", _j = _a % " + S(na) + ";");
            cg.addLine("unsigned long long _t = 0ull;");
            cg.addBlock("switch (_j)", [&]() {
                for (int j = 0; j < na; j++) {
                    const std::string src = narrow[j] ? "(unsigned long long)_kn_all[(_b * " + S(nNarrow) + " + " + S(pos[j]) + ") * " + BS
                                                      : "_kp_all[(_b * " + S(nWide) + " + " + S(pos[j]) + ") * " + BS;
                    cg.addLine("case " + S(j) + ": for (int _u = (int)(threadIdx.x & 31u); _u < (int)blockDim.x; _u += 32) _t += " +
                               src + " + _u]; break;");
                }
                cg.addLine("default: break;");
            });
            cg.addLine("#pragma unroll");
            cg.addLine("for (int _o = 16; _o > 0; _o >>= 1) _t += __shfl_xor_sync(0xffffffffu, _t, _o);");
            cg.addLine("if ((threadIdx.x & 31u) != 0u || _t == 0ull) continue;");
            cg.addLine("const long long _tot = (long long)_t;");
            cg.addBlock("switch (_j)", [&]() {
                for (int j = 0; j < na; j++) {
                    const auto& ag = aggregates_[j];
                    cg.addLine("case " + S(j) + ": " + (ag.isWide ? "gpudb_acc128_add(" : "gpudb_acc64_add(") + out +
                               " + _b * " + S(vpb) + " + " + S(ag.offset) + ", _tot); break;");
                }
                cg.addLine("default: break;");
            });
        });
    } else if (st == Strategy::Shared) {
        const int words = nb * vpb;
        const int soff = cg.allocDynamicSmem(words * 8);
        cg.addComment("keyed aggregation: per-block shared-memory table of " + S(words) + " words");
        cg.addLine("unsigned long long* _ks = reinterpret_cast<unsigned long long*>(gpudb_smem + " + S(soff) + ");");
        cg.addLine("for (int _w = threadIdx.x; _w < " + S(words) + "; _w += blockDim.x) _ks[_w] = 0ull;");
        cg.addLine("__syncthreads();");
        child_->produce(cg, [&]() {
            emitValues();
            cg.addBlock("if ((unsigned)_bucket < " + S(nb) + "u)", [&]() {
                for (int j = 0; j < na; j++) {
                    const auto& ag = aggregates_[j];
                    const std::string base = "_ks + _bucket * " + S(vpb) + " + " + S(ag.offset);
                    if (ag.isWide)
                        cg.addLine("gpudb_acc128_add(" + base + ", _kv" + S(j) + ");");
                    else
                        cg.addLine("atomicAdd(" + base + ", (unsigned long long)_kv" + S(j) + ");");
                }
            }, " else { gpudb_set_error(gpudb_err, GPUDB_ERR_BOUNDS); }");
            consume();
        });
        cg.addLine("__syncthreads();");
        cg.addBlock("for (int _w = threadIdx.x; _w < " + S(words) + "; _w += blockDim.x)", [&]() {
            cg.addLine("const unsigned long long _v = _ks[_w];");
            cg.addLine("if (_v != 0ull) atomicAdd(" + out + " + _w, _v);");
        });
    } else {
        cg.addComment("keyed aggregation: per-row global atomics");
        child_->produce(cg, [&]() {
            emitValues();
            cg.addBlock("if ((unsigned)_bucket < " + S(nb) + "u)", [&]() {
                for (int j = 0; j < na; j++) {
                    const auto& ag = aggregates_[j];
                    const std::string addr = out + " + _bucket * " + S(vpb) + " + " + S(ag.offset);
                    if (ag.atomicOp == "add")
                        cg.addLine(std::string(ag.isWide ? "gpudb_acc128_add(" : "gpudb_acc64_add(") + addr + ", _kv" +
                                   S(j) + ");");
                    else
                        cg.addLine(std::string(ag.atomicOp == "min" ? "atomicMin(" : "atomicMax(") +
                                   "reinterpret_cast<long long*>(" + addr + "), _kv" + S(j) + ");");
                }
            }, " else { gpudb_set_error(gpudb_err, GPUDB_ERR_BOUNDS); }");
            consume();
        });
    }

    std::vector<CudaResultSchema::KeyedAggSlot> slots;
    for (const auto& a : aggregates_) slots.push_back({a.name, a.offset, a.isWide, a.scaleDown});
    cg.registerKeyedAggOutput(outputArrayName_, numBuckets_, valuesPerBucket_, slots);
}

std::string CudaKeyedAgg::describe() const {
    static const char* names[] = {"auto", "registers", "shared", "global", "registers-switch", "shared-private"};
    return "KeyedAgg(" + outputArrayName_ + ", " + S(numBuckets_) + " buckets, " + S((long long)aggregates_.size()) +
           " aggs, " + names[(int)chosenStrategy()] + ") <- " + describeChain();
}

// ===================================================================
// CudaAtomicAgg
// ===================================================================
CudaAtomicAgg::CudaAtomicAgg(std::unique_ptr<CudaOperator> child, const std::string& arrayName,
                             const std::string& bucketExpr, const std::string& valueExpr,
                             const std::string& sizeExpr, const std::string& elemType)
    : CudaUnaryOperator(std::move(child)),
      arrayName_(arrayName), bucketExpr_(bucketExpr), valueExpr_(valueExpr), sizeExpr_(sizeExpr), elemType_(elemType) {}

void CudaAtomicAgg::addAggregate(const std::string& arrayName, const std::string& valueExpr) {
    extra_.push_back({arrayName, valueExpr});
}

void CudaAtomicAgg::produce(CudaCodegen& cg, ConsumerFn consume) {
    if (elemType_ != "unsigned long long")
        throw std::runtime_error("CudaAtomicAgg: only 64-bit integer accumulators are supported");
    std::vector<std::pair<std::string, std::string>> arrs{{arrayName_, valueExpr_}};
    for (const auto& e : extra_) arrs.push_back(e);
    const int na = (int)arrs.size();
    for (const auto& a : arrs) {
        if (zeroInit_)
            cg.addAtomicBufferParam(a.first, elemType_, sizeExpr_);
        else
            cg.addBufferParam(a.first, elemType_, sizeExpr_, false);
    }
    const std::string len = "len_" + arrayName_;
    cg.addBufferLengthParam(len, arrayName_);
    const int L = smemLog2_;
    const int slots = 1 << L;
    if (L > 0) {
        const int ko = cg.allocDynamicSmem(slots * 8);
        const int vo = cg.allocDynamicSmem(slots * 8 * na);
        cg.addComment("per-block shared-memory cache of hot buckets (" + S(slots) + " slots)");
        cg.addLine("unsigned long long* _ac_k = reinterpret_cast<unsigned long long*>(gpudb_smem + " + S(ko) + ");");
        cg.addLine("unsigned long long* _ac_v = reinterpret_cast<unsigned long long*>(gpudb_smem + " + S(vo) + ");");
        cg.addLine("for (int _w = threadIdx.x; _w < " + S(slots) + "; _w += blockDim.x) _ac_k[_w] = GPUDB_EMPTY64;");
        cg.addLine("for (int _w = threadIdx.x; _w < " + S(slots * na) + "; _w += blockDim.x) _ac_v[_w] = 0ull;");
        cg.addLine("__syncthreads();");
    }
    child_->produce(cg, [&]() {
        cg.addLine("const long long _ab = (long long)(" + bucketExpr_ + ");");
        for (int j = 0; j < na; j++) cg.addLine("long long _av" + S(j) + " = (long long)(" + arrs[j].second + ");");
        auto update = [&]() {
            cg.addBlock("if ((unsigned long long)_ab >= (unsigned long long)" + len + ")", [&]() {
                cg.addLine("gpudb_set_error(gpudb_err, GPUDB_ERR_BOUNDS);");
            }, " else {");
            cg.increaseIndent();
            if (L > 0) {
                cg.addLine("const int _as = gpudb_smem_ht_slot64(_ac_k, " + S(L) + ", (unsigned long long)_ab, " +
                           S(smemProbe_) + ");");
                cg.addBlock("if (_as >= 0)", [&]() {
                    for (int j = 0; j < na; j++)
                        cg.addLine("atomicAdd(_ac_v + " + S(j * slots) + " + _as, (unsigned long long)_av" + S(j) + ");");
                }, " else {");
                cg.increaseIndent();
                for (int j = 0; j < na; j++)
                    cg.addLine("atomicAdd(" + arrs[j].first + " + _ab, (unsigned long long)_av" + S(j) + ");");
                cg.decreaseIndent();
                cg.addLine("}");
            } else {
                for (int j = 0; j < na; j++)
                    cg.addLine("atomicAdd(" + arrs[j].first + " + _ab, (unsigned long long)_av" + S(j) + ");");
            }
            cg.decreaseIndent();
            cg.addLine("}");
        };
        if (warpAgg_) {
            cg.addLine("const unsigned _am = __activemask();");
            cg.addLine("const unsigned _peers = __match_any_sync(_am, (unsigned long long)_ab);");
            for (int j = 0; j < na; j++) cg.addLine("_av" + S(j) + " = gpudb_peer_sum(_am, _peers, _av" + S(j) + ");");
            cg.addIf("(int)(threadIdx.x & 31u) == __ffs(_peers) - 1", update);
        } else {
            update();
        }
        consume();
    });
    if (L > 0) {
        cg.addLine("__syncthreads();");
        cg.addBlock("for (int _w = threadIdx.x; _w < " + S(slots) + "; _w += blockDim.x)", [&]() {
            cg.addLine("const unsigned long long _k = _ac_k[_w];");
            cg.addLine("if (_k == GPUDB_EMPTY64) continue;");
            for (int j = 0; j < na; j++)
                cg.addLine("if (_ac_v[" + S(j * slots) + " + _w] != 0ull) atomicAdd(" + arrs[j].first + " + _k, _ac_v[" +
                           S(j * slots) + " + _w]);");
        });
    }
}

std::string CudaAtomicAgg::describe() const {
    return "AtomicAgg(" + arrayName_ + "[" + bucketExpr_ + "]" + (warpAgg_ ? ", warp-agg" : "") +
           (smemLog2_ ? ", smem-cache" : "") + ") <- " + describeChain();
}

// ===================================================================
// CudaAtomicCount
// ===================================================================
CudaAtomicCount::CudaAtomicCount(std::unique_ptr<CudaOperator> child, const std::string& arrayName,
                                 const std::string& bucketExpr, const std::string& sizeExpr)
    : CudaUnaryOperator(std::move(child)), arrayName_(arrayName), bucketExpr_(bucketExpr), sizeExpr_(sizeExpr) {}

void CudaAtomicCount::produce(CudaCodegen& cg, ConsumerFn consume) {
    cg.addAtomicBufferParam(arrayName_, "unsigned long long", sizeExpr_);
    cg.addBufferLengthParam("len_" + arrayName_, arrayName_);
    long long staticSize = 0;
    try {
        size_t used = 0;
        staticSize = std::stoll(sizeExpr_, &used);
        if (used != sizeExpr_.size()) staticSize = 0;
    } catch (...) {
        staticSize = 0;
    }
    const std::string arr = arrayName_;
    if (staticSize > 0 && staticSize <= 8192) {
        const std::string sz = S(staticSize);
        cg.addComment("shared-memory histogram of " + sz + " bins");
        cg.addLine("__shared__ unsigned _hist[" + sz + "];");
        cg.addLine("for (int _h = threadIdx.x; _h < " + sz + "; _h += blockDim.x) _hist[_h] = 0u;");
        cg.addLine("__syncthreads();");
        child_->produce(cg, [&]() {
            cg.addLine("const long long _hb = (long long)(" + bucketExpr_ + ");");
            cg.addLine("if ((unsigned long long)_hb < " + sz + "ull) atomicAdd(_hist + _hb, 1u); else "
                       "gpudb_set_error(gpudb_err, GPUDB_ERR_BOUNDS);");
            consume();
        });
        cg.addLine("__syncthreads();");
        cg.addLine("for (int _h = threadIdx.x; _h < " + sz + "; _h += blockDim.x) if (_hist[_h]) atomicAdd(" + arr +
                   " + _h, (unsigned long long)_hist[_h]);");
    } else {
        child_->produce(cg, [&]() {
            cg.addLine("const long long _hb = (long long)(" + bucketExpr_ + ");");
            cg.addLine("if ((unsigned long long)_hb < (unsigned long long)len_" + arr + ") atomicAdd(" + arr +
                       " + _hb, 1ull); else gpudb_set_error(gpudb_err, GPUDB_ERR_BOUNDS);");
            consume();
        });
    }
}

std::string CudaAtomicCount::describe() const { return "AtomicCount(" + arrayName_ + "[" + bucketExpr_ + "])"; }

// ===================================================================
// CudaMaterialize
// ===================================================================
CudaMaterialize::CudaMaterialize(std::unique_ptr<CudaOperator> child, const std::string& counterName,
                                 const std::string& capacityExpr)
    : CudaUnaryOperator(std::move(child)), counterName_(counterName), capacityExpr_(capacityExpr) {}

void CudaMaterialize::addColumn(const std::string& arrayName, const std::string& type, const std::string& valueExpr,
                                const std::string& displayName) {
    columns_.push_back({arrayName, type, valueExpr, displayName.empty() ? arrayName : displayName});
}

void CudaMaterialize::produce(CudaCodegen& cg, ConsumerFn consume) {
    cg.addAtomicBufferParam(counterName_, "unsigned long long", "1");
    for (const auto& c : columns_) cg.addBufferParam(c.arrayName, c.type, capacityExpr_, false);
    cg.addSizeScalarParam("cap_" + counterName_, "long long", capacityExpr_);
    if (!intermediate_) {
        cg.registerMaterializeOutput(counterName_);
        for (const auto& c : columns_) cg.registerOutputColumn(c.displayName, c.arrayName, c.type);
    }
    bool ctaBuffered = intermediate_ && !columns_.empty() && columns_.size() <= 2;
    for (const auto& c : columns_) ctaBuffered = ctaBuffered && cudaTypeBytes(c.type) == 4;
    if (ctaBuffered) {
        // 8 KB of shared memory: 2048 rows of one column or 1024 of two
        const int nc = (int)columns_.size();
        const int kBuf = 2048 / nc;
        const int bo = cg.allocDynamicSmem(kBuf * 4 * nc + 16);
        for (int k = 0; k < nc; k++)
            cg.addLine(columns_[k].type + "* _mb_buf" + S(k) + " = reinterpret_cast<" + columns_[k].type +
                       "*>(gpudb_smem + " + S(bo + k * kBuf * 4) + ");");
        cg.addLine("unsigned* _mb_n = reinterpret_cast<unsigned*>(gpudb_smem + " + S(bo + nc * kBuf * 4) + ");");
        cg.addLine("unsigned long long* _mb_base = reinterpret_cast<unsigned long long*>(gpudb_smem + " +
                   S(bo + nc * kBuf * 4 + 8) + ");");
        cg.addLine("if (threadIdx.x == 0) *_mb_n = 0u;");
        cg.addLine("__syncthreads();");
        child_->produce(cg, [&]() {
            cg.addLine("const unsigned _mp = atomicAdd(_mb_n, 1u);");
            cg.addBlock("if (_mp < " + S(kBuf) + "u)", [&]() {
                for (int k = 0; k < nc; k++)
                    cg.addLine("_mb_buf" + S(k) + "[_mp] = (" + columns_[k].type + ")(" + columns_[k].valueExpr + ");");
            }, " else {");
            cg.increaseIndent();
            cg.addComment("the CTA's buffer is full: this row goes straight to the list");
            cg.addLine("const unsigned long long _pos = atomicAdd(" + counterName_ + ", 1ull);");
            cg.addBlock("if (_pos < (unsigned long long)cap_" + counterName_ + ")", [&]() {
                for (const auto& c : columns_)
                    cg.addLine(c.arrayName + "[_pos] = (" + c.type + ")(" + c.valueExpr + ");");
            }, " else {");
            cg.increaseIndent();
            cg.addLine("gpudb_set_error(gpudb_err, GPUDB_ERR_CAPACITY);");
            cg.decreaseIndent();
            cg.addLine("}");
            cg.decreaseIndent();
            cg.addLine("}");
            consume();
        });
        cg.addComment("append this CTA's rows with one atomic");
        cg.addLine("__syncthreads();");
        cg.addBlock("", [&]() {
            cg.addLine("const unsigned _mn = min(*_mb_n, " + S(kBuf) + "u);");
            cg.addLine("if (threadIdx.x == 0) *_mb_base = _mn ? atomicAdd(" + counterName_ +
                       ", (unsigned long long)_mn) : 0ull;");
            cg.addLine("__syncthreads();");
            cg.addBlock("for (unsigned _w = threadIdx.x; _w < _mn; _w += blockDim.x)", [&]() {
                cg.addLine("const unsigned long long _pos = *_mb_base + _w;");
                cg.addBlock("if (_pos < (unsigned long long)cap_" + counterName_ + ")", [&]() {
                    for (int k = 0; k < nc; k++)
                        cg.addLine(columns_[k].arrayName + "[_pos] = _mb_buf" + S(k) + "[_w];");
                }, " else {");
                cg.increaseIndent();
                cg.addLine("gpudb_set_error(gpudb_err, GPUDB_ERR_CAPACITY);");
                cg.decreaseIndent();
                cg.addLine("}");
            });
        });
        return;
    }
    child_->produce(cg, [&]() {
        cg.addLine("const unsigned long long _pos = gpudb_warp_reserve(" + counterName_ + ", true);");
        cg.addBlock("if (_pos < (unsigned long long)cap_" + counterName_ + ")", [&]() {
            for (const auto& c : columns_)
                cg.addLine(c.arrayName + "[_pos] = (" + c.type + ")(" + c.valueExpr + ");");
        }, " else { gpudb_set_error(gpudb_err, GPUDB_ERR_CAPACITY); }");
        consume();
    });
}

std::string CudaMaterialize::describe() const {
    return "Materialize(" + S((long long)columns_.size()) + " columns) <- " + describeChain();
}

// ===================================================================
// Hash build / probe / group-by
// ===================================================================
CudaHashBuild::CudaHashBuild(std::unique_ptr<CudaOperator> child, const std::string& tableName,
                             const std::string& keyExpr, const std::string& keyType, const std::string& capacityExpr,
                             HashLayout layout, int maxProbe)
    : CudaUnaryOperator(std::move(child)),
      table_(tableName), keyExpr_(keyExpr), keyType_(keyType), capExpr_(capacityExpr), layout_(layout),
      maxProbe_(maxProbe) {}

void CudaHashBuild::addPayload(const std::string& column, const std::string& type, const std::string& valueExpr) {
    payloads_.push_back({column, type, valueExpr});
}

void CudaHashBuild::produce(CudaCodegen& cg, ConsumerFn consume) {
    const KeyOps ko = keyOps(keyType_, layout_);
    const std::string cap = hashSlotsExpr(capExpr_);
    cg.addHashMapParam(table_ + "_keys", ko.store, cap);
    for (const auto& p : payloads_) cg.addBufferParam(table_ + "_" + p.column, p.type, cap, false);
    cg.addSizeScalarParam(table_ + "_log2cap", "int", hashLog2Expr(capExpr_));
    child_->produce(cg, [&]() {
        cg.addLine("const long long _hslot = " + ko.ins + "(" + table_ + "_keys, " + table_ + "_log2cap, " + ko.cast + "(" +
                   keyExpr_ + "), " + S(probeArg(layout_, maxProbe_)) + "u, gpudb_err);");
        cg.addIf("_hslot >= 0", [&]() {
            for (const auto& p : payloads_)
                cg.addLine(table_ + "_" + p.column + "[_hslot] = (" + p.type + ")(" + p.valueExpr + ");");
            consume();
        });
    });
}

std::string CudaHashBuild::describe() const { return "HashBuild(" + table_ + ", key=" + keyExpr_ + ") <- " + describeChain(); }

CudaHashProbe::CudaHashProbe(std::unique_ptr<CudaOperator> child, const std::string& tableName,
                             const std::string& keyExpr, const std::string& keyType, const std::string& capacityExpr,
                             const std::string& slotVar, HashLayout layout, int maxProbe)
    : CudaUnaryOperator(std::move(child)),
      table_(tableName), keyExpr_(keyExpr), keyType_(keyType), capExpr_(capacityExpr), slotVar_(slotVar),
      layout_(layout), maxProbe_(maxProbe) {}

void CudaHashProbe::addPayloadRead(const std::string& column, const std::string& type) {
    payloadReads_.push_back({column, type});
}

void CudaHashProbe::produce(CudaCodegen& cg, ConsumerFn consume) {
    const KeyOps ko = keyOps(keyType_, layout_);
    cg.addHashMapReadParam(table_ + "_keys", ko.store);
    for (const auto& p : payloadReads_) cg.addReadBufferParam(table_ + "_" + p.first, p.second);
    cg.addSizeScalarParam(table_ + "_log2cap", "int", hashLog2Expr(capExpr_));
    cg.pushScanHint({CudaCodegen::ScanHint::Barrier, "", ""});
    struct Pop {
        CudaCodegen& c;
        ~Pop() { c.popScanHint(); }
    } pop{cg};
    child_->produce(cg, [&]() {
        cg.addLine("const long long " + slotVar_ + " = " + ko.find + "(" + table_ + "_keys, " + table_ + "_log2cap, " +
                   ko.cast + "(" + keyExpr_ + "), " + S(probeArg(layout_, maxProbe_)) + "u);");
        cg.addIf(slotVar_ + " >= 0", [&]() { consume(); });
    });
}

std::string CudaHashProbe::describe() const { return "HashProbe(" + table_ + ", key=" + keyExpr_ + ") <- " + describeChain(); }

CudaHashGroupBy::CudaHashGroupBy(std::unique_ptr<CudaOperator> child, const std::string& tableName,
                                 const std::string& keyExpr, const std::string& keyType,
                                 const std::string& capacityExpr, HashLayout layout, int maxProbe)
    : CudaUnaryOperator(std::move(child)),
      table_(tableName), keyExpr_(keyExpr), keyType_(keyType), capExpr_(capacityExpr), layout_(layout),
      maxProbe_(maxProbe) {}

void CudaHashGroupBy::addAggregate(const std::string& name, const std::string& valueExpr) {
    aggs_.push_back({name, valueExpr});
}

void CudaHashGroupBy::setDeviceCapacity(const std::string& groupsExpr, const std::string& boundExpr,
                                        const std::vector<std::string>& counters) {
    devGroups_ = groupsExpr;
    devBound_ = boundExpr;
    devCounters_ = counters;
}

CudaHashInit::CudaHashInit(const std::string& tableName, const std::string& keyType, HashLayout layout,
                           const std::vector<std::string>& aggNames, const std::string& groupsExpr,
                           const std::string& boundExpr, const std::vector<std::string>& counters)
    : table_(tableName), keyType_(keyType), layout_(layout), aggs_(aggNames), groups_(groupsExpr), bound_(boundExpr),
      counters_(counters) {}

// Insert `keyVar` into a group-by's main table and add `vals` to its
// aggregates. slotList: 0 none; 1 record created groups in the CTA's
// shared buffer (_gl_buf / _gl_n, overflow straight to the list); 2 append
// created groups to the global list directly.
static void emitHashMainUpdate(CudaCodegen& cg, const std::string& table, const std::string& keys, const KeyOps& ko, bool packed,
                        int strideLog2, HashLayout layout, int maxProbe, const std::vector<std::string>& aggs,
                        const std::string& keyVar, const std::vector<std::string>& vals, int slotList) {
    constexpr int kSlotBuf = 1024;
    const std::string list = table + "_slotlist", nlist = table + "_nslots";
    if (slotList) cg.addLine("bool _gnew = false;");
    cg.addLine("const long long _gslot = " + ko.ins + "(" + keys + ", " + (packed ? S(strideLog2) + ", " : "") + table +
               "_log2cap, " + ko.cast + keyVar + ", " + S(probeArg(layout, maxProbe)) + "u, gpudb_err" +
               (slotList ? ", &_gnew" : "") + ");");
    cg.addBlock("if (_gslot >= 0)", [&]() {
        for (size_t j = 0; j < aggs.size(); j++) {
            const std::string dst = packed ? keys + " + ((unsigned long long)_gslot << " + S(strideLog2) + ") + " + S(1 + j)
                                           : table + "_" + aggs[j] + " + _gslot";
            cg.addLine("atomicAdd(" + dst + ", (unsigned long long)" + vals[j] + ");");
        }
        if (slotList == 1)
            cg.addBlock("if (_gnew)", [&]() {  // group created
                cg.addLine("const unsigned _gp = atomicAdd(_gl_n, 1u);");
                cg.addLine("if (_gp < " + S(kSlotBuf) + "u) _gl_buf[_gp] = (unsigned)_gslot;");
                cg.addLine("else " + list + "[atomicAdd(" + nlist + ", 1ull)] = (unsigned)_gslot;");
            });
        else if (slotList == 2)
            cg.addLine("if (_gnew) " + list + "[atomicAdd(" + nlist + ", 1ull)] = (unsigned)_gslot;");
    });
}

void CudaHashInit::produce(CudaCodegen& cg, ConsumerFn consume) {
    const KeyOps ko = keyOps(keyType_, layout_);
    const std::string cap = hashSlotsExpr(bound_);
    cg.addBufferParam(table_ + "_keys", ko.store, cap, false, 0);
    for (const auto& a : aggs_) cg.addBufferParam(table_ + "_" + a, "unsigned long long", cap, false, 0);
    for (const auto& c : counters_) cg.addReadBufferParam(c, "unsigned long long");
    cg.addSizeScalarParam(table_ + "_log2max", "int", hashLog2Expr(bound_));
    cg.addLine("const int _hi_log2 = gpudb_device_log2cap((unsigned long long)(" + groups_ + "), " + table_ +
               "_log2max);");
    cg.addBlock("for (long long _w = tid; _w < (1ll << _hi_log2); _w += tpg)", [&]() {
        cg.addLine(table_ + "_keys[_w] = (" + ko.store + ")(~(" + ko.store + ")0);");
        for (const auto& a : aggs_) cg.addLine(table_ + "_" + a + "[_w] = 0ull;");
    });
    consume();
}

std::string CudaHashInit::describe() const { return "HashInit(" + table_ + ", slots for " + groups_ + ")"; }

void CudaHashGroupBy::produce(CudaCodegen& cg, ConsumerFn consume) {
    if (aggs_.empty()) throw std::runtime_error("CudaHashGroupBy: no aggregates");
    const KeyOps ko = keyOps(keyType_, layout_, true);
    const bool dev = !devGroups_.empty();
    const std::string cap = hashSlotsExpr(dev ? devBound_ : capExpr_);
    const bool packed = layout_ == HashLayout::Packed;
    int strideLog2 = 0;
    while ((1 << strideLog2) < 1 + (int)aggs_.size()) ++strideLog2;
    const std::string keys = packed ? table_ + "_slots" : table_ + "_keys";
    if (packed) {
        if (dev) throw std::runtime_error("CudaHashGroupBy: a device-sized table uses the linear layout");
        // word 0 of a slot holds ~key (0 = empty), the aggregates follow
        cg.addAtomicBufferParam(keys, "unsigned long long", "(" + cap + ") * " + S(1 << strideLog2));
        cg.addSizeScalarParam(table_ + "_log2cap", "int", hashLog2Expr(capExpr_));
    } else if (dev) {
        // allocated for the bound, initialised by the table's HashInit phase
        cg.addBufferParam(keys, ko.store, cap, false, 0);
        for (const auto& a : aggs_) cg.addBufferParam(table_ + "_" + a.name, "unsigned long long", cap, false, 0);
        for (const auto& c : devCounters_) cg.addReadBufferParam(c, "unsigned long long");
        cg.addSizeScalarParam(table_ + "_log2max", "int", hashLog2Expr(devBound_));
        cg.addLine("const int " + table_ + "_log2cap = gpudb_device_log2cap((unsigned long long)(" + devGroups_ + "), " +
                   table_ + "_log2max);");
    } else {
        cg.addHashMapParam(keys, ko.store, cap);
        for (const auto& a : aggs_) cg.addAtomicBufferParam(table_ + "_" + a.name, "unsigned long long", cap);
        cg.addSizeScalarParam(table_ + "_log2cap", "int", hashLog2Expr(capExpr_));
    }
    const int na = (int)aggs_.size();
    const int L = smemLog2_;
    const bool smem = L > 0 && ko.store == "unsigned long long";
    if (smem) {
        const int slots = 1 << L;
        const int ko_off = cg.allocDynamicSmem(slots * 8);
        const int vo_off = cg.allocDynamicSmem(slots * 8 * na);
        cg.addComment("per-block shared-memory pre-aggregation table (" + S(slots) + " slots) for heavy hitters");
        cg.addLine("unsigned long long* _gs_k = reinterpret_cast<unsigned long long*>(gpudb_smem + " + S(ko_off) + ");");
        cg.addLine("unsigned long long* _gs_v = reinterpret_cast<unsigned long long*>(gpudb_smem + " + S(vo_off) + ");");
        cg.addBlock("for (int _w = threadIdx.x; _w < " + S(slots) + "; _w += blockDim.x)", [&]() {
            cg.addLine("_gs_k[_w] = GPUDB_EMPTY64;");
            for (int j = 0; j < na; j++) cg.addLine("_gs_v[" + S(j) + " * " + S(slots) + " + _w] = 0ull;");
        });
        cg.addLine("__syncthreads();");
    }
    const std::string list = table_ + "_slotlist", nlist = table_ + "_nslots";
    // Groups created by this CTA are listed in shared memory first and
    // appended to the global slot list with one atomic per CTA at the end;
    // a per-group atomic on the single global counter would serialise in L2.
    constexpr int kSlotBuf = 1024;
    if (slotList_) {
        cg.addBufferParam(list, "unsigned", cap, false);
        cg.addAtomicBufferParam(nlist, "unsigned long long", "1");
        const int bo = cg.allocDynamicSmem(kSlotBuf * 4 + 16);
        cg.addLine("unsigned* _gl_buf = reinterpret_cast<unsigned*>(gpudb_smem + " + S(bo) + ");");
        cg.addLine("unsigned* _gl_n = _gl_buf + " + S(kSlotBuf) + ";");
        cg.addLine("unsigned long long* _gl_base = reinterpret_cast<unsigned long long*>(_gl_buf + " + S(kSlotBuf + 2) +
                   ");");
        cg.addLine("if (threadIdx.x == 0) *_gl_n = 0u;");
        cg.addLine("__syncthreads();");
    }
    std::vector<std::string> aggNames;
    for (const auto& a : aggs_) aggNames.push_back(a.name);
    auto mainUpdate = [&](const std::string& keyVar, const std::vector<std::string>& vals) {
        emitHashMainUpdate(cg, table_, keys, ko, packed, strideLog2, layout_, maxProbe_, aggNames, keyVar, vals,
                           slotList_ ? 1 : 0);
    };
    const bool warm = warmLog2_ > 0;
    if (warm) {
        if (dev || ko.store != "unsigned long long")
            throw std::runtime_error("CudaHashGroupBy: the warm tier needs 64-bit keys and a host-sized table");
        cg.addHashMapParam(table_ + "_wkeys", "unsigned long long", S(1ll << warmLog2_));
        for (const auto& a : aggs_) cg.addAtomicBufferParam(table_ + "_w" + a.name, "unsigned long long", S(1ll << warmLog2_));
    }
    // the warm tier first (an L2-resident table of the first keys to reach
    // it), the main table for the keys it cannot place
    auto globalUpdate = [&](const std::string& keyVar, const std::vector<std::string>& vals) {
        if (!warm) {
            mainUpdate(keyVar, vals);
            return;
        }
        cg.addLine("const long long _gws = gpudb_ht_try_insert64(" + table_ + "_wkeys, " + S(warmLog2_) +
                   ", (unsigned long long)" + keyVar + ", " + S(warmProbe_) + "u);");
        cg.addBlock("if (_gws >= 0)", [&]() {
            for (int j = 0; j < na; j++)
                cg.addLine("atomicAdd(" + table_ + "_w" + aggs_[j].name + " + _gws, (unsigned long long)" + vals[j] + ");");
        }, " else {");
        cg.increaseIndent();
        mainUpdate(keyVar, vals);
        cg.decreaseIndent();
        cg.addLine("}");
    };
    child_->produce(cg, [&]() {
        cg.addLine("const long long _gk = (long long)(" + keyExpr_ + ");");
        std::vector<std::string> vals;
        for (int j = 0; j < na; j++) {
            cg.addLine("long long _gv" + S(j) + " = (long long)(" + aggs_[j].valueExpr + ");");
            vals.push_back("_gv" + S(j));
        }
        auto update = [&]() {
            if (smem) {
                cg.addLine("const int _gss = gpudb_smem_ht_slot64(_gs_k, " + S(L) + ", (unsigned long long)_gk, " +
                           S(smemProbe_) + ");");
                cg.addBlock("if (_gss >= 0)", [&]() {
                    for (int j = 0; j < na; j++)
                        cg.addLine("atomicAdd(_gs_v + " + S(j) + " * " + S(1 << L) + " + _gss, (unsigned long long)_gv" +
                                   S(j) + ");");
                }, " else {");
                cg.increaseIndent();
                globalUpdate("(_gk)", vals);
                cg.decreaseIndent();
                cg.addLine("}");
            } else {
                globalUpdate("(_gk)", vals);
            }
        };
        if (warpAgg_) {
            cg.addLine("const unsigned _gm = __activemask();");
            cg.addLine("const unsigned _gpeers = __match_any_sync(_gm, (unsigned long long)_gk);");
            for (int j = 0; j < na; j++) cg.addLine("_gv" + S(j) + " = gpudb_peer_sum(_gm, _gpeers, _gv" + S(j) + ");");
            cg.addIf("(int)(threadIdx.x & 31u) == __ffs(_gpeers) - 1", update);
        } else {
            update();
        }
        consume();
    });
    if (smem) {
        cg.addComment("flush the shared-memory table into the global table");
        cg.addLine("__syncthreads();");
        cg.addBlock("for (int _w = threadIdx.x; _w < " + S(1 << L) + "; _w += blockDim.x)", [&]() {
            cg.addLine("const unsigned long long _fk = _gs_k[_w];");
            cg.addLine("if (_fk == GPUDB_EMPTY64) continue;");
            std::vector<std::string> vals;
            for (int j = 0; j < na; j++) vals.push_back("_gs_v[" + S(j) + " * " + S(1 << L) + " + _w]");
            globalUpdate("(_fk)", vals);
        });
    }
    if (slotList_) {
        cg.addComment("append this CTA's created groups to the global slot list");
        cg.addLine("__syncthreads();");
        cg.addBlock("", [&]() {
            cg.addLine("const unsigned _gn = min(*_gl_n, " + S(kSlotBuf) + "u);");
            cg.addLine("if (threadIdx.x == 0) *_gl_base = _gn ? atomicAdd(" + nlist + ", (unsigned long long)_gn) : 0ull;");
            cg.addLine("__syncthreads();");
            cg.addLine("for (unsigned _w = threadIdx.x; _w < _gn; _w += blockDim.x) " + list +
                       "[*_gl_base + _w] = _gl_buf[_w];");
        });
    }
    auto& hs = cg.resultSchema();
    hs.kind = CudaResultSchema::HASH_AGG;
    hs.hashAgg.keyBuffer = keys;
    hs.hashAgg.keyType = ko.store;
    hs.hashAgg.capacitySymbol = cap;
    hs.hashAgg.aggs.clear();
    for (const auto& a : aggs_) hs.hashAgg.aggs.push_back({a.name, packed ? keys : table_ + "_" + a.name});
    hs.hashAgg.packedStride = packed ? (1 << strideLog2) : 0;
}

std::string CudaHashGroupBy::describe() const {
    return "HashGroupBy(" + table_ + ", key=" + keyExpr_ +
           (layout_ == HashLayout::Bucket8 ? ", bucket8" : layout_ == HashLayout::Packed ? ", packed" : ", linear") +
           (warpAgg_ ? ", warp-agg" : "") + (smemLog2_ ? ", smem-preagg" : "") +
           (warmLog2_ ? ", warm tier " + S(1ll << warmLog2_) : "") + ") <- " + describeChain();
}

CudaHashWarmFlush::CudaHashWarmFlush(const std::string& tableName, const std::string& capacityExpr, HashLayout layout,
                                     int maxProbe, const std::vector<std::string>& aggNames, int warmLog2,
                                     bool slotList)
    : table_(tableName), capExpr_(capacityExpr), layout_(layout), maxProbe_(maxProbe), aggs_(aggNames),
      warmLog2_(warmLog2), slotList_(slotList) {}

void CudaHashWarmFlush::produce(CudaCodegen& cg, ConsumerFn consume) {
    const KeyOps ko = keyOps("long long", layout_, true);
    const std::string cap = hashSlotsExpr(capExpr_);
    const bool packed = layout_ == HashLayout::Packed;
    int strideLog2 = 0;
    while ((1 << strideLog2) < 1 + (int)aggs_.size()) ++strideLog2;
    const std::string keys = packed ? table_ + "_slots" : table_ + "_keys";
    // the main table as the group-by phase left it: no fill here
    if (packed) {
        cg.addBufferParam(keys, "unsigned long long", "(" + cap + ") * " + S(1 << strideLog2), false, 0);
    } else {
        cg.addBufferParam(keys, ko.store, cap, false, 0);
        for (const auto& a : aggs_) cg.addBufferParam(table_ + "_" + a, "unsigned long long", cap, false, 0);
    }
    cg.addSizeScalarParam(table_ + "_log2cap", "int", hashLog2Expr(capExpr_));
    if (slotList_) {
        cg.addBufferParam(table_ + "_slotlist", "unsigned", cap, false, 0);
        cg.addBufferParam(table_ + "_nslots", "unsigned long long", "1", false, 0);
    }
    cg.addReadBufferParam(table_ + "_wkeys", "unsigned long long");
    for (const auto& a : aggs_) cg.addReadBufferParam(table_ + "_w" + a, "unsigned long long");
    cg.addComment("every warm entry into the main table");
    cg.addBlock("for (long long _w = tid; _w < " + S(1ll << warmLog2_) + "ll; _w += tpg)", [&]() {
        cg.addLine("const unsigned long long _wk = " + table_ + "_wkeys[_w];");
        cg.addLine("if (_wk == GPUDB_EMPTY64) continue;");
        std::vector<std::string> vals;
        for (const auto& a : aggs_) vals.push_back(table_ + "_w" + a + "[_w]");
        emitHashMainUpdate(cg, table_, keys, ko, packed, strideLog2, layout_, maxProbe_, aggs_, "(long long)_wk", vals,
                           slotList_ ? 2 : 0);
    });
    consume();
}

std::string CudaHashWarmFlush::describe() const {
    return "HashWarmFlush(" + table_ + ", " + S(1ll << warmLog2_) + " warm slots)";
}

// ===================================================================
// CudaTopK
// ===================================================================
CudaTopK::CudaTopK(std::unique_ptr<CudaOperator> child, const std::string& outPrefix, const std::string& keyExpr,
                   const std::string& valueExpr, int k, int maxBlocks)
    : CudaUnaryOperator(std::move(child)), out_(outPrefix), keyExpr_(keyExpr), valueExpr_(valueExpr), k_(k),
      maxBlocks_(maxBlocks) {}

void CudaTopK::produce(CudaCodegen& cg, ConsumerFn consume) {
    if (k_ < 1 || k_ > 32) throw std::runtime_error("CudaTopK: k must be in [1,32]");
    const std::string K = S(k_);
    cg.setPhaseMaxThreadgroups(maxBlocks_);
    cg.addBufferParam(out_ + "_keys", "long long", K, true, 0);
    cg.addBufferParam(out_ + "_vals", "long long", K, true, 0);
    cg.addAtomicBufferParam(out_ + "_count", "unsigned long long", "1");
    cg.addBufferParam(out_ + "_pkeys", "long long", S((long long)k_ * maxBlocks_), false);
    cg.addBufferParam(out_ + "_pvals", "long long", S((long long)k_ * maxBlocks_), false);
    cg.addAtomicBufferParam(out_ + "_ticket", "unsigned", "1");
    if (auto* list = dynamic_cast<CudaSlotListScan*>(child_.get())) {
        produceOverList(cg, *list, consume);
        return;
    }
    cg.addLine("long long _tk_v[" + K + "], _tk_k[" + K + "];");
    cg.addLine("#pragma unroll");
    cg.addLine("for (int _q = 0; _q < " + K + "; ++_q) { _tk_v[_q] = GPUDB_TOPK_NONE_VAL; _tk_k[_q] = GPUDB_TOPK_NONE_KEY; }");
    child_->produce(cg, [&]() {
        cg.addLine("gpudb_topk_push<" + K + ">(_tk_v, _tk_k, (long long)(" + valueExpr_ + "), (long long)(" + keyExpr_ +
                   "));");
        consume();
    });
    cg.addComment("block merge (warp shuffle merge, then warp 0 over the warps' lists), per-block list to global,"
                  " then the last block merges all per-block lists the same way");
    cg.addLine("long long _tw_v[" + K + "], _tw_k[" + K + "];");
    cg.addLine("__shared__ long long _ts_v[32 * " + K + "], _ts_k[32 * " + K + "];");
    cg.addLine("__shared__ bool _t_last;");
    // every thread's (_tk_v, _tk_k) list -> warp 0 holds the block's best K in (_tw_v, _tw_k)
    auto blockMerge = [&]() {
        cg.addLine("gpudb_topk_warp_merge<" + K + ">(_tk_v, _tk_k, _tw_v, _tw_k);");
        cg.addBlock("if ((threadIdx.x & 31u) == 0u)", [&]() {
            cg.addLine("#pragma unroll");
            cg.addLine("for (int _q = 0; _q < " + K + "; ++_q) { _ts_v[(threadIdx.x >> 5) * " + K + " + _q] = _tw_v[_q]; "
                       "_ts_k[(threadIdx.x >> 5) * " + K + " + _q] = _tw_k[_q]; }");
        });
        cg.addLine("__syncthreads();");
        cg.addBlock("if (threadIdx.x < 32u)", [&]() {
            cg.addLine("#pragma unroll");
            cg.addLine("for (int _q = 0; _q < " + K + "; ++_q) { _tk_v[_q] = GPUDB_TOPK_NONE_VAL; _tk_k[_q] = GPUDB_TOPK_NONE_KEY; }");
            cg.addLine("for (int _e = (int)threadIdx.x; _e < (int)(blockDim.x >> 5) * " + K + "; _e += 32) gpudb_topk_push<" +
                       K + ">(_tk_v, _tk_k, _ts_v[_e], _ts_k[_e]);");
            cg.addLine("gpudb_topk_warp_merge<" + K + ">(_tk_v, _tk_k, _tw_v, _tw_k);");
        });
    };
    blockMerge();
    cg.addBlock("if (threadIdx.x == 0u)", [&]() {
        cg.addLine("for (int _q = 0; _q < " + K + "; ++_q) { " + out_ + "_pvals[blockIdx.x * " + K + " + _q] = _tw_v[_q]; " +
                   out_ + "_pkeys[blockIdx.x * " + K + " + _q] = _tw_k[_q]; }");
        cg.addLine("__threadfence();");
        cg.addLine("_t_last = (atomicAdd(" + out_ + "_ticket, 1u) == gridDim.x - 1u);");
    });
    cg.addLine("__syncthreads();");
    cg.addBlock("if (_t_last)", [&]() {
        cg.addLine("__threadfence();");
        cg.addLine("#pragma unroll");
        cg.addLine("for (int _q = 0; _q < " + K + "; ++_q) { _tk_v[_q] = GPUDB_TOPK_NONE_VAL; _tk_k[_q] = GPUDB_TOPK_NONE_KEY; }");
        cg.addLine("for (int _e = (int)threadIdx.x; _e < (int)gridDim.x * " + K + "; _e += (int)blockDim.x) gpudb_topk_push<" +
                   K + ">(_tk_v, _tk_k, __ldcg(" + out_ + "_pvals + _e), __ldcg(" + out_ + "_pkeys + _e));");
        blockMerge();
        cg.addBlock("if (threadIdx.x == 0u)", [&]() {
            cg.addLine("unsigned long long _cnt = 0ull;");
            cg.addBlock("for (int _q = 0; _q < " + K + "; ++_q)", [&]() {
                cg.addLine("if (_tw_k[_q] == GPUDB_TOPK_NONE_KEY && _tw_v[_q] == GPUDB_TOPK_NONE_VAL) break;");
                cg.addLine(out_ + "_vals[_q] = _tw_v[_q]; " + out_ + "_keys[_q] = _tw_k[_q]; ++_cnt;");
            });
            cg.addLine(out_ + "_count[0] = _cnt;");
            cg.addLine(out_ + "_ticket[0] = 0u;  // self-reset for the next launch");
        });
    });
    auto& rs = cg.resultSchema();
    rs.kind = CudaResultSchema::TOPK;
    rs.topk.keyBuffer = out_ + "_keys";
    rs.topk.valueBuffer = out_ + "_vals";
    rs.topk.countBuffer = out_ + "_count";
    rs.topk.k = k_;
}

// Top-k over a slot list (the groups a hash group-by created): every warp
// walks the list 32 entries at a time and keeps its best K one per lane
// (lane j holds the j-th best), so a thread carries two values instead of
// two K-lists and an entry costs one ballot unless it beats the warp's
// K-th best. Warps' lists meet in shared memory, blocks' lists in global
// memory, and the last block to finish merges those the same way. A full
// list's K-th value is a floor: K entries are at least that good, so an
// entry valued below the highest such floor cannot enter and is never
// offered to the block and grid merges (values equal to it still are).
void CudaTopK::produceOverList(CudaCodegen& cg, const CudaSlotListScan& list, ConsumerFn consume) {
    const std::string K = S(k_);
    const std::string n = list.declareList(cg);
    const std::string& i = list.indexVar();
    // highest full-list floor of all blocks, as value ^ sign bit (0 = none)
    cg.addAtomicBufferParam(out_ + "_floor", "unsigned long long", "1");
    cg.addLine("const int _tl = (int)(threadIdx.x & 31u);");
    cg.addLine("long long _tr_v = GPUDB_TOPK_NONE_VAL, _tr_k = GPUDB_TOPK_NONE_KEY;");
    cg.addLine("const long long _tl_n = " + n + ";");
    cg.addBlock("for (long long _tb = (tid >> 5) * 32; _tb < _tl_n; _tb += (tpg >> 5) * 32)", [&]() {
        cg.addLine("long long _tc_v = GPUDB_TOPK_NONE_VAL, _tc_k = GPUDB_TOPK_NONE_KEY;");
        cg.addBlock("if (_tb + _tl < _tl_n)", [&]() {
            cg.addLine("const long long " + i + " = (long long)__ldcg(" + list.listBuffer() + " + _tb + _tl);");
            cg.addLine("const long long _row = " + i + "; (void)_row;");
            cg.addLine("_tc_v = (long long)(" + valueExpr_ + ");");
            cg.addLine("_tc_k = (long long)(" + keyExpr_ + ");");
            consume();
        });
        cg.addLine("gpudb_topk_warp_offer<" + K + ">(_tr_v, _tr_k, _tc_v, _tc_k);");
    });
    cg.addLine("__shared__ long long _ts_v[32 * 32], _ts_k[32 * 32];");
    cg.addLine("__shared__ bool _t_last;");
    // (the biased floor of a full list, or 0)
    const std::string fullFloor = "(_tl == " + S(k_ - 1) + " && !(_tr_k == GPUDB_TOPK_NONE_KEY && _tr_v == "
                                  "GPUDB_TOPK_NONE_VAL) ? ((unsigned long long)_tr_v ^ 0x8000000000000000ull) : 0ull)";
    // every warp's sorted list -> warp 0 holds the block's best K: a tree of
    // pairwise list merges through shared memory, log2(warps) levels
    auto blockMerge = [&]() {
        cg.addLine("_ts_v[threadIdx.x] = _tr_v; _ts_k[threadIdx.x] = _tr_k;");
        cg.addBlock("for (int _ts = 1; _ts < (int)(blockDim.x >> 5); _ts <<= 1)", [&]() {
            cg.addLine("__syncthreads();");
            cg.addLine("const int _tw = (int)(threadIdx.x >> 5);");
            cg.addBlock("if ((_tw & (2 * _ts - 1)) == 0 && _tw + _ts < (int)(blockDim.x >> 5))", [&]() {
                cg.addLine("gpudb_topk_warp_merge_list<" + K + ">(_tr_v, _tr_k, _ts_v[(_tw + _ts) * 32 + _tl], "
                           "_ts_k[(_tw + _ts) * 32 + _tl]);");
                cg.addLine("_ts_v[threadIdx.x] = _tr_v; _ts_k[threadIdx.x] = _tr_k;");
            });
        });
        cg.addLine("__syncthreads();");
    };
    blockMerge();
    cg.addBlock("if (threadIdx.x < 32u)", [&]() {
        cg.addBlock("if (_tl < " + K + ")", [&]() {
            cg.addLine(out_ + "_pvals[blockIdx.x * " + K + " + _tl] = _tr_v;");
            cg.addLine(out_ + "_pkeys[blockIdx.x * " + K + " + _tl] = _tr_k;");
            cg.addLine("const unsigned long long _fl = " + fullFloor + ";");
            cg.addLine("if (_fl) atomicMax(" + out_ + "_floor, _fl);");
            cg.addLine("__threadfence();");
        });
        cg.addLine("__syncwarp();");
        cg.addLine("if (_tl == 0) _t_last = (atomicAdd(" + out_ + "_ticket, 1u) == gridDim.x - 1u);");
    });
    cg.addLine("__syncthreads();");
    cg.addBlock("if (_t_last)", [&]() {
        cg.addLine("__threadfence();");
        cg.addLine("_tr_v = GPUDB_TOPK_NONE_VAL; _tr_k = GPUDB_TOPK_NONE_KEY;");
        cg.addLine("const long long _tgf = (long long)(__ldcg(" + out_ + "_floor) ^ 0x8000000000000000ull);");
        // each warp merges whole block lists (lane j loads a list's j-th
        // entry), four lists' loads in flight before any merge; a list with
        // no entry at or above the highest block floor cannot contribute
        cg.addLine("const int _tnw = (int)(blockDim.x >> 5);");
        cg.addBlock("for (int _b0 = (int)(threadIdx.x >> 5); _b0 < (int)gridDim.x; _b0 += 4 * _tnw)", [&]() {
            cg.addLine("long long _ev[4], _ek[4];");
            cg.addLine("#pragma unroll");
            cg.addBlock("for (int _u = 0; _u < 4; ++_u)", [&]() {
                cg.addLine("const int _b = _b0 + _u * _tnw;");
                cg.addLine("const bool _tin = _b < (int)gridDim.x && _tl < " + K + ";");
                cg.addLine("_ev[_u] = _tin ? __ldcg(" + out_ + "_pvals + _b * " + K + " + _tl) : GPUDB_TOPK_NONE_VAL;");
                cg.addLine("_ek[_u] = _tin ? __ldcg(" + out_ + "_pkeys + _b * " + K + " + _tl) : GPUDB_TOPK_NONE_KEY;");
            });
            cg.addLine("#pragma unroll");
            cg.addBlock("for (int _u = 0; _u < 4; ++_u)", [&]() {
                cg.addLine("const bool _tok = _ev[_u] >= _tgf && !(_ev[_u] == GPUDB_TOPK_NONE_VAL && "
                           "_ek[_u] == GPUDB_TOPK_NONE_KEY);");
                cg.addLine("if (__any_sync(0xffffffffu, _tok)) gpudb_topk_warp_merge_list<" + K +
                           ">(_tr_v, _tr_k, _ev[_u], _ek[_u]);");
            });
        });
        blockMerge();
        cg.addBlock("if (threadIdx.x < 32u)", [&]() {
            cg.addLine("const bool _tf = _tl < " + K + " && !(_tr_k == GPUDB_TOPK_NONE_KEY && _tr_v == GPUDB_TOPK_NONE_VAL);");
            cg.addLine("const unsigned _tm = __ballot_sync(0xffffffffu, _tf);");
            cg.addLine("if (_tf) { " + out_ + "_vals[_tl] = _tr_v; " + out_ + "_keys[_tl] = _tr_k; }");
            cg.addBlock("if (_tl == 0)", [&]() {
                cg.addLine(out_ + "_count[0] = (unsigned long long)__popc(_tm);");
                cg.addLine(out_ + "_ticket[0] = 0u;  // self-reset for the next launch");
                cg.addLine(out_ + "_floor[0] = 0ull;");
            });
        });
    });
    auto& rs = cg.resultSchema();
    rs.kind = CudaResultSchema::TOPK;
    rs.topk.keyBuffer = out_ + "_keys";
    rs.topk.valueBuffer = out_ + "_vals";
    rs.topk.countBuffer = out_ + "_count";
    rs.topk.k = k_;
}

std::string CudaTopK::describe() const {
    return "TopK(k=" + S(k_) + ", key=" + keyExpr_ + ", value=" + valueExpr_ + ") <- " + describeChain();
}

// ===================================================================
// CudaSortPass
// ===================================================================
CudaSortPass::CudaSortPass(Mode mode, const std::string& prefix, const std::string& countBuffer,
                           const std::string& capacityExpr, int pass)
    : mode_(mode), prefix_(prefix), count_(countBuffer), cap_(capacityExpr), pass_(pass) {}

void CudaSortPass::setInput(const std::string& keys, const std::string& counts, const std::string& values) {
    inK_ = keys;
    inC_ = counts;
    inV_ = values;
}

void CudaSortPass::setOutputNames(const std::string& key, const std::string& count, const std::string& value) {
    outK_ = key;
    outC_ = count;
    outV_ = value;
}

void CudaSortPass::produce(CudaCodegen& cg, ConsumerFn consume) {
    (void)consume;
    const int bs = cg.currentThreadgroupSize();
    if (kChunk % bs != 0) throw std::runtime_error("CudaSortPass: the block size must divide 2048");
    const std::string CH = S(kChunk), VT = S(kChunk / bs), P = prefix_;
    const std::string kMax = "0x7fffffffffffffffll", kMin = "(-0x7fffffffffffffffll - 1ll)";
    cg.addReadBufferParam(count_, "unsigned long long");
    cg.addSizeScalarParam("cap_" + P, "long long", cap_);
    auto set = [&](int which, bool write) {
        for (const char* c : {"k", "c", "v"}) {
            const std::string n = P + "_" + c + S(which);
            if (write) cg.addBufferParam(n, "long long", cap_, false);
            else cg.addReadBufferParam(n, "long long");
        }
    };
    cg.addLine("const long long _sn = min((long long)__ldcg(" + count_ + "), cap_" + P + ");");
    cg.addLine("const int _sneed = gpudb_merge_passes(_sn, " + CH + ");");
    if (mode_ == Mode::Chunks) {
        cg.addReadBufferParam(inK_, "long long");
        cg.addReadBufferParam(inC_, "long long");
        cg.addReadBufferParam(inV_, "long long");
        set(0, true);
        const int off = cg.allocDynamicSmem(3 * kChunk * 8);
        cg.addComment("sort " + CH + "-row chunks in shared memory (bitonic network), value desc, key asc");
        cg.addLine("long long* _sk = reinterpret_cast<long long*>(gpudb_smem + " + S(off) + ");");
        cg.addLine("long long* _sv = _sk + " + CH + ";");
        cg.addLine("long long* _sc = _sv + " + CH + ";");
        cg.addBlock("for (long long _t = blockIdx.x; _t * " + CH + "ll < _sn; _t += gridDim.x)", [&]() {
            cg.addLine("const long long _b = _t * " + CH + "ll;");
            cg.addBlock("for (int _e = threadIdx.x; _e < " + CH + "; _e += blockDim.x)", [&]() {
                cg.addLine("const long long _r = _b + _e;");
                cg.addLine("if (_r < _sn) { _sk[_e] = " + inK_ + "[_r]; _sv[_e] = " + inV_ + "[_r]; _sc[_e] = " + inC_ +
                           "[_r]; } else { _sk[_e] = " + kMax + "; _sv[_e] = " + kMin + "; _sc[_e] = 0ll; }");
            });
            cg.addLine("__syncthreads();");
            cg.addBlock("for (int _size = 2; _size <= " + CH + "; _size <<= 1)", [&]() {
                cg.addBlock("for (int _st = _size >> 1; _st > 0; _st >>= 1)", [&]() {
                    cg.addBlock("for (int _e = threadIdx.x; _e < " + S(kChunk / 2) + "; _e += blockDim.x)", [&]() {
                        cg.addLine("const int _i = 2 * _e - (_e & (_st - 1)), _j = _i + _st;");
                        cg.addLine("const bool _up = (_i & _size) == 0;");
                        cg.addLine("const bool _jb = gpudb_row_before(_sv[_j], _sk[_j], _sv[_i], _sk[_i]);");
                        cg.addBlock("if (_up ? _jb : !_jb)", [&]() {
                            cg.addLine("long long _x = _sk[_i]; _sk[_i] = _sk[_j]; _sk[_j] = _x;");
                            cg.addLine("_x = _sv[_i]; _sv[_i] = _sv[_j]; _sv[_j] = _x;");
                            cg.addLine("_x = _sc[_i]; _sc[_i] = _sc[_j]; _sc[_j] = _x;");
                        });
                    });
                    cg.addLine("__syncthreads();");
                });
            });
            cg.addBlock("for (int _e = threadIdx.x; _e < " + CH + "; _e += blockDim.x)", [&]() {
                cg.addLine("const long long _r = _b + _e;");
                cg.addLine("if (_r < _sn) { " + P + "_k0[_r] = _sk[_e]; " + P + "_v0[_r] = _sv[_e]; " + P +
                           "_c0[_r] = _sc[_e]; }");
            });
            cg.addLine("__syncthreads();");
        });
    } else if (mode_ == Mode::Merge) {
        const int src = pass_ & 1, dst = src ^ 1;
        set(src, false);
        set(dst, true);
        const std::string SR = P + "_", SS = S(src), DS = S(dst);
        const int off = cg.allocDynamicSmem(3 * kChunk * 8);
        cg.addComment("merge pass " + S(pass_) + ": runs of " + CH + " << " + S(pass_) + " rows merge pairwise");
        cg.addLine("if (" + S(pass_) + " >= _sneed) return;  // the runs already cover all rows");
        cg.addLine("long long* _sk = reinterpret_cast<long long*>(gpudb_smem + " + S(off) + ");");
        cg.addLine("long long* _sv = _sk + " + CH + ";");
        cg.addLine("long long* _sc = _sv + " + CH + ";");
        cg.addLine("__shared__ int _ssplit[2];");
        cg.addLine("const long long _L = " + CH + "ll << " + S(pass_) + ";");
        cg.addBlock("for (long long _t = blockIdx.x; _t * " + CH + "ll < _sn; _t += gridDim.x)", [&]() {
            cg.addLine("const long long _o0 = _t * " + CH + "ll, _base = (_o0 / (2 * _L)) * (2 * _L);");
            cg.addLine("const long long _aB = _base, _aE = min(_base + _L, _sn), _bE = min(_base + 2 * _L, _sn);");
            cg.addLine("const int _na = (int)(_aE - _aB), _nb = (int)(_bE - _aE);");
            cg.addLine("const int _d0 = (int)(_o0 - _base), _d1 = (int)(min(_o0 + " + CH + "ll, _bE) - _base);");
            cg.addComment("the tile's split of the two runs: warps 0 and 1 search its two diagonals");
            cg.addBlock("if (threadIdx.x < 64u)", [&]() {
                cg.addLine("const int _sp = gpudb_merge_path_warp(" + SR + "v" + SS + " + _aB, " + SR + "k" + SS +
                           " + _aB, _na, " + SR + "v" + SS + " + _aE, " + SR + "k" + SS + " + _aE, _nb, threadIdx.x < 32u ? _d0 : _d1);");
                cg.addLine("if ((threadIdx.x & 31u) == 0u) _ssplit[threadIdx.x >> 5] = _sp;");
            });
            cg.addLine("__syncthreads();");
            cg.addLine("const int _a0 = _ssplit[0], _a1 = _ssplit[1], _b0 = _d0 - _a0, _b1 = _d1 - _a1;");
            cg.addLine("const int _ca = _a1 - _a0, _cb = _b1 - _b0, _tot = _ca + _cb;");
            cg.addBlock("for (int _e = threadIdx.x; _e < _tot; _e += blockDim.x)", [&]() {
                cg.addLine("const long long _r = _e < _ca ? _aB + _a0 + _e : _aE + _b0 + (_e - _ca);");
                cg.addLine("_sk[_e] = " + SR + "k" + SS + "[_r]; _sv[_e] = " + SR + "v" + SS + "[_r]; _sc[_e] = " + SR +
                           "c" + SS + "[_r];");
            });
            cg.addLine("__syncthreads();");
            cg.addBlock("", [&]() {
                cg.addLine("const int _dd = (int)threadIdx.x * " + VT + ";");
                cg.addBlock("if (_dd < _tot)", [&]() {
                    cg.addLine("int _ia = gpudb_merge_path(_sv, _sk, _ca, _sv + _ca, _sk + _ca, _cb, _dd), _ib = _dd - _ia;");
                    cg.addBlock("for (int _q = 0; _q < " + VT + " && _dd + _q < _tot; ++_q)", [&]() {
                        cg.addLine("const bool _ta = _ib >= _cb || (_ia < _ca && !gpudb_row_before(_sv[_ca + _ib], "
                                   "_sk[_ca + _ib], _sv[_ia], _sk[_ia]));");
                        cg.addLine("const int _x = _ta ? _ia++ : _ca + _ib++;");
                        cg.addLine("const long long _w = _o0 + _dd + _q;");
                        cg.addLine(SR + "k" + DS + "[_w] = _sk[_x]; " + SR + "v" + DS + "[_w] = _sv[_x]; " + SR + "c" + DS +
                                   "[_w] = _sc[_x];");
                    });
                });
            });
            cg.addLine("__syncthreads();");
        });
    } else {
        set(0, false);
        set(1, false);
        const std::string n = P + "_n";
        cg.addAtomicBufferParam(n, "unsigned long long", "1");
        cg.addBufferParam(P + "_out_k", "long long", cap_, false);
        cg.addBufferParam(P + "_out_c", "long long", cap_, false);
        cg.addBufferParam(P + "_out_v", "long long", cap_, false);
        cg.addComment("the sorted rows, in order, from the buffer set the last merge pass wrote");
        cg.addLine("const long long* _ok = (_sneed & 1) ? " + P + "_k1 : " + P + "_k0;");
        cg.addLine("const long long* _oc = (_sneed & 1) ? " + P + "_c1 : " + P + "_c0;");
        cg.addLine("const long long* _ov = (_sneed & 1) ? " + P + "_v1 : " + P + "_v0;");
        cg.addBlock("for (long long _r = tid; _r < _sn; _r += tpg)", [&]() {
            cg.addLine(P + "_out_k[_r] = _ok[_r]; " + P + "_out_c[_r] = _oc[_r]; " + P + "_out_v[_r] = _ov[_r];");
        });
        cg.addLine("if (tid == 0) " + n + "[0] = (unsigned long long)_sn;");
        cg.registerMaterializeOutput(n);
        cg.registerOutputColumn(outK_, P + "_out_k", "long long");
        cg.registerOutputColumn(outC_, P + "_out_c", "long long");
        cg.registerOutputColumn(outV_, P + "_out_v", "long long");
    }
}

std::string CudaSortPass::describe() const {
    switch (mode_) {
        case Mode::Chunks: return "SortChunks(" + prefix_ + ", " + S(kChunk) + " rows, value desc, key asc)";
        case Mode::Merge: return "SortMerge(" + prefix_ + ", pass " + S(pass_) + ")";
        default: return "SortEmit(" + prefix_ + ")";
    }
}

}  // namespace gpudb
