#include "cuda_codegen.h"

#include <sstream>
#include <stdexcept>

namespace gpudb {

// The device template library, embedded at build time from gpudb_device.cuh.
static const char kDeviceHeader[] =
#include "device_header_gen.inc"
    ;

const char* CudaCodegen::deviceHeader() { return kDeviceHeader; }

CudaCodegen::PhaseInfo& CudaCodegen::cur(const char* op) {
    if (current_ < 0) throw std::runtime_error(std::string("CudaCodegen::") + op + ": no active phase");
    return phases_[current_];
}

// ---------------------------------------------------------------------------
// emission
// ---------------------------------------------------------------------------
void CudaCodegen::addLine(const std::string& line) { cur("addLine").code += indent() + line + "\n"; }

void CudaCodegen::addBlock(const std::string& header, const std::function<void()>& body,
                           const std::string& trailing) {
    cur("addBlock").code += indent() + header + " {\n";
    indentLevel_++;
    body();
    indentLevel_--;
    cur("addBlock").code += indent() + "}" + trailing + "\n";
}

void CudaCodegen::addIf(const std::string& condition, const std::function<void()>& body) {
    addBlock("if (" + condition + ")", body);
}

void CudaCodegen::addComment(const std::string& comment) { cur("addComment").code += indent() + "// " + comment + "\n"; }
void CudaCodegen::increaseIndent() { indentLevel_++; }
void CudaCodegen::decreaseIndent() {
    if (indentLevel_ > 0) indentLevel_--;
}
void CudaCodegen::addRawCode(const std::string& code) { cur("addRawCode").code += code; }
void CudaCodegen::addHelper(const std::string& code) { helperCode_ += code + "\n"; }
std::string CudaCodegen::fresh(const std::string& stem) { return stem + std::to_string(freshCounter_++); }

int CudaCodegen::pushScanHint(const ScanHint& h) {
    scanHints_.push_back(h);
    return (int)scanHints_.size() - 1;
}

void CudaCodegen::popScanHint() {
    if (!scanHints_.empty()) {
        prefetchVars_.erase((int)scanHints_.size() - 1);
        scanHints_.pop_back();
    }
}

void CudaCodegen::setPrefetchVar(int id, const std::string& var) {
    if (var.empty()) prefetchVars_.erase(id);
    else prefetchVars_[id] = var;
}

std::string CudaCodegen::prefetchVar(int id) const {
    auto it = prefetchVars_.find(id);
    return it == prefetchVars_.end() ? std::string() : it->second;
}

// ---------------------------------------------------------------------------
// phases
// ---------------------------------------------------------------------------
void CudaCodegen::beginPhase(const std::string& phaseName) {
    if (current_ >= 0)
        throw std::runtime_error("CudaCodegen::beginPhase: previous phase '" + phases_[current_].name +
                                 "' not ended");
    for (const auto& p : phases_)
        if (p.name == phaseName) throw std::runtime_error("CudaCodegen::beginPhase: duplicate phase '" + phaseName + "'");
    phases_.push_back({});
    current_ = (int)phases_.size() - 1;
    phases_.back().name = phaseName;
    indentLevel_ = 1;
}

void CudaCodegen::endPhase() {
    cur("endPhase");
    current_ = -1;
    indentLevel_ = 1;
}

void CudaCodegen::setPhaseScannedTable(const std::string& t) { cur("setPhaseScannedTable").scannedTable = t; }
void CudaCodegen::setPhaseThreadgroupSize(int s) {
    if (s <= 0 || s > 1024 || (s % 32) != 0)
        throw std::runtime_error("setPhaseThreadgroupSize: block size must be a multiple of 32 in [32,1024]");
    cur("setPhaseThreadgroupSize").threadgroupSize = s;
}
void CudaCodegen::setPhaseSingleThread(bool s) { cur("setPhaseSingleThread").isSingleThread = s; }
void CudaCodegen::setPhaseMaxThreadgroups(int m) { cur("setPhaseMaxThreadgroups").maxThreadgroups = m; }
void CudaCodegen::setPhaseDynamicSmem(int b) { cur("setPhaseDynamicSmem").dynamicSmemBytes = b; }
void CudaCodegen::setPhaseTileRows(int r) { cur("setPhaseTileRows").tileRows = r; }
void CudaCodegen::setPhaseRowsPerThread(int r) { cur("setPhaseRowsPerThread").rowsPerThread = r > 0 ? r : 1; }
void CudaCodegen::setPhaseMinBlocksPerSM(int n) { cur("setPhaseMinBlocksPerSM").minBlocksPerSM = n > 0 ? n : 1; }
void CudaCodegen::setPhaseSmemCarveout(int percent) { cur("setPhaseSmemCarveout").smemCarveout = percent; }
int CudaCodegen::currentThreadgroupSize() const {
    if (current_ < 0) throw std::runtime_error("currentThreadgroupSize: no active phase");
    return phases_[current_].threadgroupSize;
}

// ---------------------------------------------------------------------------
// bindings
// ---------------------------------------------------------------------------
void CudaCodegen::pushBinding(const char* op, CudaParamBinding b, bool dedup) {
    auto& ph = cur(op);
    for (const auto& e : ph.bindings) {
        if (e.name != b.name) continue;
        if (e.kind != b.kind || e.elementType != b.elementType)
            throw std::runtime_error(std::string(op) + ": conflicting redeclaration of '" + b.name + "' in phase '" +
                                     ph.name + "'");
        // One argument per name per kernel. `dedup` documents the caller's
        // intent (the reference dedups buffers but not columns); CUDA
        // forbids duplicate parameter names, so both are folded here.
        (void)dedup;
        return;
    }
    if (!b.sizeExpr.empty() && b.kind == CudaParamKind::DeviceBuffer && !b.readOnly)
        globalBufferSizes_[b.name] = b.sizeExpr;
    ph.bindings.push_back(std::move(b));
}

void CudaCodegen::addColumnParam(const std::string& paramName, const std::string& elemType,
                                 const std::string& tableName, bool late) {
    CudaParamBinding b;
    b.late = late;
    b.name = paramName;
    b.cudaTypeDecl = "const " + elemType + "* __restrict__";
    b.kind = CudaParamKind::TableData;
    b.tableName = tableName.empty() ? paramName : tableName;
    b.elementType = elemType;
    b.readOnly = true;
    pushBinding("addColumnParam", std::move(b), false);
}

void CudaCodegen::addTableSizeParam(const std::string& table) {
    CudaParamBinding b;
    b.name = tableSizeName(table);
    b.cudaTypeDecl = "long long";
    b.kind = CudaParamKind::TableSize;
    b.tableName = table;
    b.elementType = "long long";
    pushBinding("addTableSizeParam", std::move(b), false);
}

void CudaCodegen::addBufferParam(const std::string& name, const std::string& elemType,
                                 const std::string& sizeExpr, bool zeroInit, int fillByte) {
    CudaParamBinding b;
    b.name = name;
    b.cudaTypeDecl = elemType + "* __restrict__";
    b.kind = CudaParamKind::DeviceBuffer;
    b.elementType = elemType;
    b.sizeExpr = sizeExpr;
    b.zeroInit = zeroInit;
    b.fillByte = fillByte;
    pushBinding("addBufferParam", std::move(b), true);
}

void CudaCodegen::addReadBufferParam(const std::string& name, const std::string& elemType) {
    CudaParamBinding b;
    b.name = name;
    b.cudaTypeDecl = "const " + elemType + "* __restrict__";
    b.kind = CudaParamKind::DeviceBuffer;
    b.elementType = elemType;
    b.readOnly = true;
    pushBinding("addReadBufferParam", std::move(b), true);
}

void CudaCodegen::addAtomicBufferParam(const std::string& name, const std::string& elemType,
                                       const std::string& sizeExpr) {
    addBufferParam(name, elemType, sizeExpr, true, 0);
}

void CudaCodegen::addScalarParam(const std::string& name, const std::string& type) {
    CudaParamBinding b;
    b.name = name;
    b.cudaTypeDecl = type;
    b.kind = CudaParamKind::ConstantScalar;
    b.elementType = type;
    pushBinding("addScalarParam", std::move(b), true);
}

void CudaCodegen::addSizeScalarParam(const std::string& name, const std::string& type,
                                     const std::string& sizeExpr) {
    CudaParamBinding b;
    b.name = name;
    b.cudaTypeDecl = type;
    b.kind = CudaParamKind::ConstantScalar;
    b.elementType = type;
    b.sizeExpr = sizeExpr;
    pushBinding("addSizeScalarParam", std::move(b), true);
}

void CudaCodegen::addBufferLengthParam(const std::string& name, const std::string& bufferName) {
    CudaParamBinding b;
    b.name = name;
    b.cudaTypeDecl = "long long";
    b.kind = CudaParamKind::BufferLength;
    b.elementType = "long long";
    b.tableName = bufferName;
    pushBinding("addBufferLengthParam", std::move(b), true);
}

int CudaCodegen::allocDynamicSmem(int bytes) {
    auto& ph = cur("allocDynamicSmem");
    const int off = (ph.dynamicSmemBytes + 127) & ~127;
    ph.dynamicSmemBytes = off + ((bytes + 127) & ~127);
    return off;
}

void CudaCodegen::addConstantDataParam(const std::string& name, const std::string& type, size_t bytes) {
    CudaParamBinding b;
    b.name = name;
    b.cudaTypeDecl = "const " + type + "* __restrict__";
    b.kind = CudaParamKind::ConstantData;
    b.elementType = type;
    b.hostCopyBytes = bytes;
    b.readOnly = true;
    pushBinding("addConstantDataParam", std::move(b), false);
}

void CudaCodegen::addBitmapReadParam(const std::string& name, const std::string& sizeExpr) {
    (void)sizeExpr;  // sized by the phase that builds it
    addReadBufferParam(name, "unsigned");
}

void CudaCodegen::addBitmapWriteParam(const std::string& name, const std::string& sizeExpr) {
    addBufferParam(name, "unsigned", sizeExpr, true, 0);
}

void CudaCodegen::addHashMapParam(const std::string& keysName, const std::string& keyType,
                                  const std::string& capacityExpr) {
    addBufferParam(keysName, keyType, capacityExpr, true, 0xFF);
}

void CudaCodegen::addHashMapReadParam(const std::string& keysName, const std::string& keyType) {
    addReadBufferParam(keysName, keyType);
}

void CudaCodegen::setBufferSize(const std::string& name, const std::string& sizeExpr) {
    globalBufferSizes_[name] = sizeExpr;
}

// ---------------------------------------------------------------------------
// result schema
// ---------------------------------------------------------------------------
void CudaCodegen::registerScalarAggColumn(const std::string& displayName, const std::string& buffer,
                                          bool isWide, int scaleDown) {
    resultSchema_.kind = CudaResultSchema::SCALAR_AGG;
    resultSchema_.scalarAggs.push_back({displayName, buffer, isWide, scaleDown});
}

void CudaCodegen::registerMaterializeOutput(const std::string& counterBuffer) {
    resultSchema_.kind = CudaResultSchema::MATERIALIZE;
    resultSchema_.counterBuffer = counterBuffer;
}

void CudaCodegen::registerOutputColumn(const std::string& displayName, const std::string& bufferName,
                                       const std::string& elementType) {
    resultSchema_.columns.push_back({displayName, bufferName, elementType});
}

void CudaCodegen::registerKeyedAggOutput(const std::string& bufferName, int numBuckets, int valuesPerBucket,
                                         const std::vector<CudaResultSchema::KeyedAggSlot>& slots) {
    resultSchema_.kind = CudaResultSchema::KEYED_AGG;
    resultSchema_.keyedAgg.bufferName = bufferName;
    resultSchema_.keyedAgg.numBuckets = numBuckets;
    resultSchema_.keyedAgg.valuesPerBucket = valuesPerBucket;
    resultSchema_.keyedAgg.slots = slots;
}

// ---------------------------------------------------------------------------
// print
// ---------------------------------------------------------------------------
void CudaCodegen::assignArgIndices(PhaseInfo& phase) {
    bool hasErr = false;
    for (const auto& b : phase.bindings)
        if (b.kind == CudaParamKind::ErrorWord) hasErr = true;
    if (!hasErr) {
        CudaParamBinding e;
        e.name = "gpudb_err";
        e.cudaTypeDecl = "unsigned* __restrict__";
        e.kind = CudaParamKind::ErrorWord;
        e.elementType = "unsigned";
        phase.bindings.push_back(e);
    }
    int i = 0;
    for (auto& b : phase.bindings) b.argIndex = i++;
}

std::string CudaCodegen::generateSignature(const PhaseInfo& phase) const {
    std::ostringstream s;
    const int bs = phase.isSingleThread ? 32 : phase.threadgroupSize;
    s << "extern \"C\" __global__ void __launch_bounds__(" << bs << ", " << phase.minBlocksPerSM << ")\n"
      << phase.name << "(\n";
    for (size_t i = 0; i < phase.bindings.size(); i++) {
        const auto& b = phase.bindings[i];
        s << "    " << b.cudaTypeDecl << " " << b.name << (i + 1 < phase.bindings.size() ? "," : "") << "\n";
    }
    s << ")";
    return s.str();
}

std::string CudaCodegen::print() {
    if (current_ >= 0) throw std::runtime_error("CudaCodegen::print: phase '" + phases_[current_].name + "' not ended");
    std::ostringstream out;
    out << kDeviceHeader << "\n";
    if (!helperCode_.empty()) out << "// --- plan helpers ---\n" << helperCode_ << "\n";
    for (size_t pi = 0; pi < phases_.size(); pi++) {
        assignArgIndices(phases_[pi]);
        const auto& ph = phases_[pi];
        out << "\n// === Phase " << pi << ": " << ph.name << " ===\n";
        out << generateSignature(ph) << " {\n";
        out << "    GPUDB_THREAD_VARS\n";
        if (ph.dynamicSmemBytes > 0) out << "    extern __shared__ __align__(1024) unsigned char gpudb_smem[];\n";
        out << ph.code;
        out << "}\n";
    }
    return out.str();
}

std::vector<CudaParamBinding> CudaCodegen::getAllBindings() const {
    std::vector<CudaParamBinding> all;
    std::unordered_set<std::string> seen;
    for (const auto& ph : phases_)
        for (const auto& b : ph.bindings)
            if (seen.insert(b.name).second) all.push_back(b);
    return all;
}

}  // namespace gpudb
