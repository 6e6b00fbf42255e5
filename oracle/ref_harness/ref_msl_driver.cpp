// ref_msl_driver.cpp — TEST INFRASTRUCTURE (oracle pinning).
//
// Linked against the reference engine's own planning layer and operator
// emitters (codegen/planning/metal_plan_builder.cpp,
// codegen/operators/metal_operators.cpp, codegen/core/metal_codegen_base.cpp,
// codegen/core/metal_param_binding.cpp, compiled unmodified from the
// reference tree by build_ref.py). It asks the reference to generate the MSL
// kernels for the benchmark pipelines and writes:
//   <out>/ref_<plan>.cpp   the reference's MSL, made compilable as C++ with
//                          msl_cpu_shim.h, plus an extern "C" launcher per
//                          phase taking the kernel's [[buffer(N)]] arguments
//                          as void* in index order;
//   <out>/manifest.json    per plan: phases, bindings (name, type, kind,
//                          size expression, fill), result schema.
//
// Plans:
//   Q1  buildMetalPlan(analyzed Q1 shape, "Q1")  with ship_day <= 2436
//   Q6  buildMetalPlan(analyzed Q6 shape, "Q6")  with the config constants
//   JOIN  the reference's Q3 operator chain (BitmapBuild -> BitmapProbe ->
//         AtomicAgg, metal_plan_builder.cpp:1170-1239) over the join
//         configuration's columns
//   GROUPBY the reference's AtomicAgg + AtomicCount (Q18 / Q13 operators)
//         grouping by rank % card
//   ANTI / HIST / DIRECT  the reference's Q22 anti-join, Q13 count histogram
//         and Q3 direct-address join chains over the join configuration
//   Q5  buildMetalPlan(empty analysis, "Q5"): the reference's own five-phase
//         multi-join (metal_plan_builder.cpp:894-1015), reached by name
#include <fstream>
#include <iostream>
#include <regex>
#include <sstream>
#include <string>

#include "metal_plan_builder.h"

using namespace codegen;

namespace {

ExprPtr col(const std::string& c, DataType t) { return Expr::col("lineitem", c, 0, t); }

SelectTarget sumOf(ExprPtr e, const std::string& alias) {
    SelectTarget t;
    t.isAgg = true;
    t.alias = alias;
    AggTarget a;
    a.func = AggFunc::SUM;
    a.innerExpr = e;
    a.alias = alias;
    t.agg = a;
    t.expr = e;
    return t;
}

AnalyzedQuery q1Query() {
    AnalyzedQuery aq;
    aq.tables = {"lineitem"};
    aq.filters = {Predicate::cmp(CmpOp::LE, col("l_shipdate", DataType::DATE), Expr::lit(2436))};
    aq.groupBy = {col("l_returnflag", DataType::CHAR1), col("l_linestatus", DataType::CHAR1)};
    auto one = Expr::litf(1.0f);
    auto price = col("l_extendedprice", DataType::FLOAT);
    auto disc = col("l_discount", DataType::FLOAT);
    auto discPrice = Expr::binary(ExprOp::MUL, price, Expr::binary(ExprOp::SUB, one, disc));
    aq.targets = {sumOf(col("l_quantity", DataType::FLOAT), "sum_qty"), sumOf(price, "sum_base_price"),
                  sumOf(discPrice, "sum_disc_price"),
                  sumOf(Expr::binary(ExprOp::MUL, discPrice,
                                     Expr::binary(ExprOp::ADD, one, col("l_tax", DataType::FLOAT))),
                        "sum_charge")};
    return aq;
}

AnalyzedQuery q6Query() {
    AnalyzedQuery aq;
    aq.tables = {"lineitem"};
    auto ship = col("l_shipdate", DataType::DATE);
    aq.filters = {Predicate::cmp(CmpOp::GE, ship, Expr::lit(365)), Predicate::cmp(CmpOp::LT, ship, Expr::lit(730)),
                  Predicate::between(col("l_discount", DataType::FLOAT), Expr::litf(0.05f), Expr::litf(0.07f)),
                  Predicate::cmp(CmpOp::LT, col("l_quantity", DataType::FLOAT), Expr::lit(24))};
    aq.targets = {sumOf(Expr::binary(ExprOp::MUL, col("l_extendedprice", DataType::FLOAT),
                                     col("l_discount", DataType::FLOAT)),
                        "revenue")};
    return aq;
}

MetalQueryPlan::Phase makePhase(const std::string& name, std::unique_ptr<MetalOperator> root, int tg) {
    MetalQueryPlan::Phase p;
    p.name = name;
    p.root = std::move(root);
    p.threadgroupSize = tg;
    return p;
}

MetalQueryPlan joinPlan() {
    MetalQueryPlan plan;
    plan.name = "JOIN";
    {
        auto scan = std::make_unique<MetalGridStrideScan>("dim", "row", "i");
        scan->addColumn("b_key", "int");
        scan->addColumn("b_order_day", "int");
        scan->addColumn("b_segment", "char");
        auto sel = std::make_unique<MetalSelection>(std::move(scan), "b_segment[i] == 1 && b_order_day[i] < 1170");
        auto bm = std::make_unique<MetalBitmapBuild>(std::move(sel), "d_jb_bitmap", "b_key[i]", "(maxKey + 31) / 32");
        plan.phases.push_back(makePhase("JOIN_build_bitmap", std::move(bm), 256));
    }
    {
        auto scan = std::make_unique<MetalGridStrideScan>("probe", "row", "i");
        scan->addColumn("p_fk", "int");
        scan->addColumn("p_ship_day", "int");
        scan->addColumn("p_price", "float");
        scan->addColumn("p_discount", "float");
        auto sel = std::make_unique<MetalSelection>(std::move(scan), "p_ship_day[i] > 1170");
        auto pr = std::make_unique<MetalBitmapProbe>(std::move(sel), "d_jb_bitmap", "p_fk[i]");
        auto agg = std::make_unique<MetalAtomicAgg>(std::move(pr), "d_revenue", "p_fk[i]",
                                                    "p_price[i] * (1.0f - p_discount[i])", "maxKey", "atomic_float",
                                                    "float");
        plan.phases.push_back(makePhase("JOIN_probe_aggregate", std::move(agg), 1024));
    }
    return plan;
}

// The same join with its matching probe rows written out by the
// reference's Materialize operator (metal_operators.cpp:618-643): row id,
// key and revenue per match, at atomic output positions.
MetalQueryPlan joinRowsPlan() {
    MetalQueryPlan plan;
    plan.name = "JOINROWS";
    {
        auto scan = std::make_unique<MetalGridStrideScan>("dim", "row", "i");
        scan->addColumn("b_key", "int");
        scan->addColumn("b_order_day", "int");
        scan->addColumn("b_segment", "char");
        auto sel = std::make_unique<MetalSelection>(std::move(scan), "b_segment[i] == 1 && b_order_day[i] < 1170");
        auto bm = std::make_unique<MetalBitmapBuild>(std::move(sel), "d_jb_bitmap", "b_key[i]", "(maxKey + 31) / 32");
        plan.phases.push_back(makePhase("JOINROWS_build_bitmap", std::move(bm), 256));
    }
    {
        auto scan = std::make_unique<MetalGridStrideScan>("probe", "row", "i");
        scan->addColumn("p_fk", "int");
        scan->addColumn("p_ship_day", "int");
        scan->addColumn("p_price", "float");
        scan->addColumn("p_discount", "float");
        auto sel = std::make_unique<MetalSelection>(std::move(scan), "p_ship_day[i] > 1170");
        auto pr = std::make_unique<MetalBitmapProbe>(std::move(sel), "d_jb_bitmap", "p_fk[i]");
        auto mt = std::make_unique<MetalMaterialize>(std::move(pr), "d_jr_n", "1");
        mt->addColumn("d_jr_row", "uint", "(uint)i", "row", "n_probe");
        mt->addColumn("d_jr_key", "int", "p_fk[i]", "key", "n_probe");
        mt->addColumn("d_jr_rev", "float", "p_price[i] * (1.0f - p_discount[i])", "revenue", "n_probe");
        plan.phases.push_back(makePhase("JOINROWS_probe_materialize", std::move(mt), 1024));
    }
    return plan;
}

MetalQueryPlan groupbyPlan() {
    MetalQueryPlan plan;
    plan.name = "GROUPBY";
    auto scan = std::make_unique<MetalGridStrideScan>("mix", "row", "i");
    scan->addColumn("m_rank_u", "int");
    scan->addColumn("m_filter", "int");
    scan->addColumn("m_value", "float");
    auto sel = std::make_unique<MetalSelection>(std::move(scan), "m_filter[i] < thr");
    auto key = std::make_unique<MetalComputeExpr>(std::move(sel), "_k", "int", "m_rank_u[i] % card");
    auto sum = std::make_unique<MetalAtomicAgg>(std::move(key), "d_sum", "_k", "m_value[i]", "card", "atomic_float",
                                                "float");
    auto cnt = std::make_unique<MetalAtomicCount>(std::move(sum), "d_cnt", "_k", "card");
    auto p = makePhase("GROUPBY_aggregate", std::move(cnt), 1024);
    p.scalarParams = {{"thr", "int"}, {"card", "int"}};
    plan.phases.push_back(std::move(p));
    return plan;
}

// The reference's anti-join operators (Q22 / Q21 use AntiBitmapProbe,
// metal_operators.cpp:157-165): probe rows whose key is NOT in the build
// side's qualifying set, binned by discount (ComputeExpr) into a float sum
// of price and a count per bin (AtomicAgg + AtomicCount).
MetalQueryPlan antiPlan() {
    MetalQueryPlan plan;
    plan.name = "ANTI";
    {
        auto scan = std::make_unique<MetalGridStrideScan>("dim", "row", "i");
        scan->addColumn("b_key", "int");
        scan->addColumn("b_order_day", "int");
        scan->addColumn("b_segment", "char");
        auto sel = std::make_unique<MetalSelection>(std::move(scan), "b_segment[i] == 1 && b_order_day[i] < 1170");
        auto bm = std::make_unique<MetalBitmapBuild>(std::move(sel), "d_ab_bitmap", "b_key[i]", "(maxKey + 31) / 32");
        plan.phases.push_back(makePhase("ANTI_build_bitmap", std::move(bm), 256));
    }
    {
        auto scan = std::make_unique<MetalGridStrideScan>("probe", "row", "i");
        scan->addColumn("p_fk", "int");
        scan->addColumn("p_ship_day", "int");
        scan->addColumn("p_price", "float");
        scan->addColumn("p_discount", "int");
        auto sel = std::make_unique<MetalSelection>(std::move(scan), "p_ship_day[i] > 1170");
        auto ap = std::make_unique<MetalAntiBitmapProbe>(std::move(sel), "d_ab_bitmap", "p_fk[i]");
        auto bin = std::make_unique<MetalComputeExpr>(std::move(ap), "_bin", "int", "p_discount[i]");
        auto sum = std::make_unique<MetalAtomicAgg>(std::move(bin), "d_a_sum", "_bin", "p_price[i]", "11",
                                                    "atomic_float", "float");
        auto cnt = std::make_unique<MetalAtomicCount>(std::move(sum), "d_a_cnt", "_bin", "11");
        plan.phases.push_back(makePhase("ANTI_probe_bins", std::move(cnt), 1024));
    }
    return plan;
}

// The reference's count histogram (Q13: AtomicCount per key, then per
// build row an ArrayLookup of its key's count into AtomicCount bins,
// metal_plan_builder.cpp:1244-1299).
MetalQueryPlan histPlan() {
    MetalQueryPlan plan;
    plan.name = "HIST";
    {
        auto scan = std::make_unique<MetalGridStrideScan>("probe", "row", "i");
        scan->addColumn("p_fk", "int");
        scan->addColumn("p_ship_day", "int");
        auto sel = std::make_unique<MetalSelection>(std::move(scan), "p_ship_day[i] > 1170");
        auto cnt = std::make_unique<MetalAtomicCount>(std::move(sel), "d_h_cnt", "p_fk[i]", "maxKey");
        plan.phases.push_back(makePhase("HIST_count", std::move(cnt), 1024));
    }
    {
        auto scan = std::make_unique<MetalGridStrideScan>("dim", "row", "i");
        scan->addColumn("b_key", "int");
        auto lk = std::make_unique<MetalArrayLookup>(std::move(scan), "d_h_cnt", "b_key[i]", "_c", "int", -1);
        auto hist = std::make_unique<MetalAtomicCount>(std::move(lk), "d_h_hist", "_c", "256");
        plan.phases.push_back(makePhase("HIST_bins", std::move(hist), 256));
    }
    return plan;
}

// The reference's direct-address join (Q3: ArrayStore of the qualifying
// build keys' order_day, then the probe's ArrayLookup and AtomicAgg,
// metal_plan_builder.cpp:1189-1236).
MetalQueryPlan directPlan() {
    MetalQueryPlan plan;
    plan.name = "DIRECT";
    {
        auto scan = std::make_unique<MetalGridStrideScan>("dim", "row", "i");
        scan->addColumn("b_key", "int");
        scan->addColumn("b_order_day", "int");
        scan->addColumn("b_segment", "char");
        auto sel = std::make_unique<MetalSelection>(std::move(scan), "b_segment[i] == 1 && b_order_day[i] < 1170");
        auto st = std::make_unique<MetalArrayStore>(std::move(sel), "d_d_day", "b_key[i]", "b_order_day[i]", "int",
                                                    "maxKey");
        plan.phases.push_back(makePhase("DIRECT_build_map", std::move(st), 256));
    }
    {
        auto scan = std::make_unique<MetalGridStrideScan>("probe", "row", "i");
        scan->addColumn("p_fk", "int");
        scan->addColumn("p_ship_day", "int");
        scan->addColumn("p_price", "float");
        scan->addColumn("p_discount", "float");
        auto sel = std::make_unique<MetalSelection>(std::move(scan), "p_ship_day[i] > 1170");
        auto lk = std::make_unique<MetalArrayLookup>(std::move(sel), "d_d_day", "p_fk[i]", "_od", "int", -1);
        auto agg = std::make_unique<MetalAtomicAgg>(std::move(lk), "d_d_rev", "p_fk[i]",
                                                    "p_price[i] * (1.0f - p_discount[i])", "maxKey", "atomic_float",
                                                    "float");
        plan.phases.push_back(makePhase("DIRECT_probe_aggregate", std::move(agg), 1024));
    }
    return plan;
}

std::string jsonEscape(const std::string& s) {
    std::string o;
    for (char c : s) {
        if (c == '"' || c == '\\') o += '\\';
        if (c == '\n') {
            o += "\\n";
            continue;
        }
        o += c;
    }
    return o;
}

const char* kindName(MetalParamKind k) {
    switch (k) {
        case MetalParamKind::TableData: return "TableData";
        case MetalParamKind::TableSize: return "TableSize";
        case MetalParamKind::DeviceBuffer: return "DeviceBuffer";
        case MetalParamKind::ConstantScalar: return "ConstantScalar";
        case MetalParamKind::ConstantData: return "ConstantData";
    }
    return "?";
}

// MSL declaration -> C++ type for the launcher cast.
std::string cppType(std::string decl) {
    for (const char* q : {"device ", "constant ", "threadgroup "}) {
        size_t p;
        while ((p = decl.find(q)) != std::string::npos) decl.erase(p, std::string(q).size());
    }
    return decl;
}

// Make the reference's MSL compilable as C++ with msl_cpu_shim.h.
std::string toCpp(const std::string& msl) {
    std::string s = msl;
    // drop the Metal preamble (the shim provides namespace metal)
    s = std::regex_replace(s, std::regex("#include <metal_stdlib>\\n"), "");
    s = std::regex_replace(s, std::regex("using namespace metal;\\n"), "");
    // `threadgroup T name[N];` statements in kernel bodies: one instance per
    // threadgroup in flight on a host thread
    s = std::regex_replace(s, std::regex("(^|\\n)(\\s*)threadgroup\\s+(\\w+\\s+\\w+\\s*\\[)"),
                           "$1$2static thread_local $3");
    // the remaining uses are pointer qualifiers
    s = std::regex_replace(s, std::regex("\\bthreadgroup\\s+(?=[A-Za-z_])"), "");
    return s;
}

void emitPlan(const MetalQueryPlan& plan, const std::string& outDir, std::ostream& manifest, bool first) {
    MetalCodegen cg = generateFromPlan(plan);
    const std::string msl = cg.print();
    std::ostringstream cpp;
    cpp << "// generated from the reference engine's code generator (plan " << plan.name << "); do not edit\n"
        << "#include \"msl_cpu_shim.h\"\nusing namespace metal;\n\n"
        << toCpp(msl) << "\n";
    for (const auto& ph : cg.getPhases()) {
        cpp << "extern \"C\" void ref_" << ph.name << "(void** a, unsigned numTG, unsigned tgSize) {\n"
            << "    metal::cpu::dispatch(numTG, tgSize, [&](uint tid, uint tpg, uint lid, uint tgs, uint gid, uint lane, "
               "uint sid) {\n"
            << "        " << ph.name << "(";
        for (size_t i = 0; i < ph.bindings.size(); i++) {
            const auto& b = ph.bindings[i];
            std::string t = cppType(b.metalTypeDecl);
            if (!t.empty() && t.back() == '&') {
                t.pop_back();
                cpp << "*(" << t << "*)a[" << b.bufferIndex << "], ";
            } else {
                cpp << "(" << t << ")a[" << b.bufferIndex << "], ";
            }
        }
        cpp << "tid, tpg, lid, tgs, gid, lane, sid);\n    });\n}\n";
    }
    std::ofstream(outDir + "/ref_" + plan.name + ".cpp") << cpp.str();

    const auto& rs = cg.getResultSchema();
    manifest << (first ? "" : ",\n") << "  \"" << plan.name << "\": {\n    \"phases\": [\n";
    const auto& phases = cg.getPhases();
    for (size_t p = 0; p < phases.size(); p++) {
        const auto& ph = phases[p];
        manifest << "      {\"name\": \"" << ph.name << "\", \"threadgroupSize\": " << ph.threadgroupSize
                 << ", \"maxThreadgroups\": " << ph.maxThreadgroups << ", \"scannedTable\": \"" << ph.scannedTable
                 << "\", \"bindings\": [";
        for (size_t i = 0; i < ph.bindings.size(); i++) {
            const auto& b = ph.bindings[i];
            manifest << (i ? ", " : "") << "{\"name\": \"" << b.name << "\", \"decl\": \"" << b.metalTypeDecl
                     << "\", \"kind\": \"" << kindName(b.kind) << "\", \"table\": \"" << b.tableName
                     << "\", \"elem\": \"" << b.elementType << "\", \"size\": \"" << jsonEscape(b.sizeExpr)
                     << "\", \"zeroInit\": " << (b.zeroInit ? "true" : "false") << ", \"fill\": " << b.fillByte
                     << ", \"index\": " << b.bufferIndex << "}";
        }
        manifest << "]}" << (p + 1 < phases.size() ? "," : "") << "\n";
    }
    manifest << "    ],\n    \"schema\": {\"kind\": " << (int)rs.kind << ", \"keyed\": {\"buffer\": \""
             << rs.keyedAgg.bufferName << "\", \"numBuckets\": " << rs.keyedAgg.numBuckets
             << ", \"valuesPerBucket\": " << rs.keyedAgg.valuesPerBucket << ", \"slots\": [";
    for (size_t i = 0; i < rs.keyedAgg.slots.size(); i++) {
        const auto& sl = rs.keyedAgg.slots[i];
        manifest << (i ? ", " : "") << "{\"name\": \"" << sl.name << "\", \"offset\": " << sl.offset
                 << ", \"isLongPair\": " << (sl.isLongPair ? "true" : "false") << ", \"scaleDown\": " << sl.scaleDown
                 << "}";
    }
    manifest << "]}, \"scalar\": [";
    for (size_t i = 0; i < rs.scalarAggs.size(); i++) {
        const auto& e = rs.scalarAggs[i];
        manifest << (i ? ", " : "") << "{\"name\": \"" << e.displayName << "\", \"lo\": \"" << e.loBuffer
                 << "\", \"hi\": \"" << e.hiBuffer << "\", \"isLongPair\": " << (e.isLongPair ? "true" : "false")
                 << ", \"scaleDown\": " << e.scaleDown << "}";
    }
    manifest << "]},\n    \"msl_chars\": " << msl.size() << "\n  }";
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) {
        std::cerr << "usage: ref_msl_driver <out_dir>\n";
        return 2;
    }
    const std::string out = argv[1];
    std::ofstream manifest(out + "/manifest.json");
    manifest << "{\n";
    auto q1 = buildMetalPlan(q1Query(), "Q1");
    auto q6 = buildMetalPlan(q6Query(), "Q6");
    auto q5 = buildMetalPlan(AnalyzedQuery{}, "Q5");
    if (!q1 || !q6 || !q5) {
        std::cerr << "reference planner did not accept the Q1/Q6/Q5 shapes\n";
        return 1;
    }
    emitPlan(*q1, out, manifest, true);
    emitPlan(*q6, out, manifest, false);
    emitPlan(joinPlan(), out, manifest, false);
    emitPlan(joinRowsPlan(), out, manifest, false);
    emitPlan(groupbyPlan(), out, manifest, false);
    emitPlan(antiPlan(), out, manifest, false);
    emitPlan(histPlan(), out, manifest, false);
    emitPlan(directPlan(), out, manifest, false);
    q5->name = "Q5";
    emitPlan(*q5, out, manifest, false);
    manifest << "\n}\n";
    std::cout << "wrote " << out << "/ref_{Q1,Q6,JOIN,JOINROWS,GROUPBY,ANTI,HIST,DIRECT,Q5}.cpp and manifest.json\n";
    return 0;
}
