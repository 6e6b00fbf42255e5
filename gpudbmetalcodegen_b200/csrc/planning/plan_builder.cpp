#include "plan_builder.h"

#include "query_ir.h"

#include <algorithm>
#include <cctype>
#include <set>
#include <sstream>
#include <stdexcept>

namespace gpudb {

// ===================================================================
// Catalog
// ===================================================================
namespace {

std::vector<TableDef> buildCatalog() {
    return {
        // Fact table (lineitem role): config-0 schema.
        {"fact",
         {{"f_ship_day", "int"},
          {"f_quantity", "long long"},
          {"f_price", "long long", 2},
          {"f_discount", "long long", 2},
          {"f_tax", "long long", 2},
          {"f_flag_a", "unsigned char", 0, "ANR"},
          {"f_flag_b", "unsigned char", 0, "FO"}}},
        // Build side (orders role): unique int keys.
        {"dim", {{"b_key", "int"}, {"b_order_day", "int"}, {"b_segment", "unsigned char"}}},
        // Probe side (lineitem role for the join).
        {"probe", {{"p_fk", "int"}, {"p_ship_day", "int"}, {"p_price", "long long", 2}, {"p_discount", "long long", 2}}},
        // Skewed-key probe / group-by input.
        {"zprobe", {{"z_key", "long long"}, {"z_value", "long long"}}},
        // Skewed-key build side: every distinct key once.
        {"zbuild", {{"zb_key", "long long"}, {"zb_payload", "int"}}},
        // Mixed-workload table: keys by rank (uniform / Zipf), filter, value.
        {"mix",
         {{"m_rank_u", "int"},
          {"m_rank_z", "int"},
          {"m_filter", "int"},
          {"m_value", "long long"},
          {"m_fk", "int"}}},
        // Mixed-workload dimension (join-agg build side).
        {"mixdim", {{"md_key", "int"}, {"md_attr", "int"}}},
        // The multi-join snowflake (the reference's Q5 shape): nation ->
        // customer / supplier -> orders -> lines.
        {"nation", {{"n_key", "int"}, {"n_region", "int"}}},
        {"cust", {{"c_key", "int"}, {"c_nation", "int"}}},
        {"supp", {{"s_key", "int"}, {"s_nation", "int"}}},
        {"ord", {{"o_key", "int"}, {"o_cust", "int"}, {"o_day", "int"}}},
        {"line", {{"l_okey", "int"}, {"l_supp", "int"}, {"l_price", "long long", 2}, {"l_discount", "long long", 2}}},
    };
}

const std::vector<TableDef>& catalog() {
    static const std::vector<TableDef> c = buildCatalog();
    return c;
}

}  // namespace

const ColumnDef& TableDef::col(const std::string& n) const {
    for (const auto& c : columns)
        if (c.name == n) return c;
    throw std::runtime_error("catalog: table '" + name + "' has no column '" + n + "'");
}

const TableDef& catalogTable(const std::string& table) {
    for (const auto& t : catalog())
        if (t.name == table) return t;
    throw std::runtime_error("catalog: unknown table '" + table + "'");
}

std::vector<std::string> catalogTables() {
    std::vector<std::string> out;
    for (const auto& t : catalog()) out.push_back(t.name);
    return out;
}

// ===================================================================
// Spec / tune parsing
// ===================================================================
SpecMap parseSpec(const std::string& spec) {
    SpecMap m;
    std::stringstream ss(spec);
    std::string item;
    while (std::getline(ss, item, ';')) {
        const auto b = item.find_first_not_of(" \t");
        if (b == std::string::npos) continue;
        item = item.substr(b, item.find_last_not_of(" \t") - b + 1);
        const auto eq = item.find('=');
        if (eq == std::string::npos) throw std::runtime_error("spec: expected key=value, got '" + item + "'");
        m[item.substr(0, eq)] = item.substr(eq + 1);
    }
    return m;
}

std::string canonicalSpec(const SpecMap& m) {
    std::string s;
    for (const auto& [k, v] : m) s += (s.empty() ? "" : ";") + k + "=" + v;
    return s;
}

std::string TuneConfig::toString() const {
    std::ostringstream o;
    o << "bs=" << blockSize << ";scan=" << (scan.mode == ScanConfig::TmaBulk ? "tma" : "direct")
      << ";tile=" << scan.tileRows << ";stages=" << scan.stages
      << ";layout="
      << (hashLayout == HashLayout::Bucket8 ? "bucket8" : hashLayout == HashLayout::Packed ? "packed" : "linear")
      << ";smem=" << smemPreAggLog2
      << ";warp=" << (warpAggregate ? 1 : 0) << ";keyed=" << keyedStrategy << ";probe=" << maxProbe
      << ";late=" << (lateMaterialize ? 1 : 0) << ";occ=" << minBlocksPerSM << ";pf=" << scan.prefetchRows << ";vec=" << scan.vectorRows << ";l2pf=" << scan.l2Prefetch
      << ";split=" << (splitJoin ? 1 : 0) << ";sprobe=" << smemProbe << ";carve=" << smemCarveout << ";bbs=" << buildBlockSize
      << ";bvec=" << buildVectorRows << ";htf=" << hashFill << ";warm=" << warmLog2 << ";wprobe=" << warmProbe
      << ";tkb=" << topkBlocks;
    return o.str();
}

TuneConfig TuneConfig::forBuild() const {
    TuneConfig t = *this;
    if (buildBlockSize > 0) t.blockSize = buildBlockSize;
    if (buildVectorRows > 0) t.scan.vectorRows = buildVectorRows;
    return t;
}

TuneConfig TuneConfig::parse(const std::string& s) {
    TuneConfig t;
    for (const auto& [k, v] : parseSpec(s)) {
        if (k == "bs") t.blockSize = std::stoi(v);
        else if (k == "scan") {
            if (v == "tma") t.scan.mode = ScanConfig::TmaBulk;
            else if (v == "direct") t.scan.mode = ScanConfig::Direct;
            else throw std::runtime_error("tune: scan must be tma|direct");
        } else if (k == "tile") t.scan.tileRows = std::stoi(v);
        else if (k == "stages") t.scan.stages = std::stoi(v);
        else if (k == "layout") {
            if (v == "linear") t.hashLayout = HashLayout::Linear;
            else if (v == "bucket8") t.hashLayout = HashLayout::Bucket8;
            else if (v == "packed") t.hashLayout = HashLayout::Packed;
            else throw std::runtime_error("tune: layout must be linear|bucket8|packed");
        } else if (k == "smem") t.smemPreAggLog2 = std::stoi(v);
        else if (k == "warp") t.warpAggregate = std::stoi(v) != 0;
        else if (k == "keyed") t.keyedStrategy = std::stoi(v);
        else if (k == "probe") t.maxProbe = std::stoi(v);
        else if (k == "late") t.lateMaterialize = std::stoi(v) != 0;
        else if (k == "occ") t.minBlocksPerSM = std::stoi(v);
        else if (k == "pf") t.scan.prefetchRows = std::stoi(v);
        else if (k == "vec") t.scan.vectorRows = std::stoi(v);
        else if (k == "l2pf") t.scan.l2Prefetch = std::stoi(v);
        else if (k == "split") t.splitJoin = std::stoi(v) != 0;
        else if (k == "carve") t.smemCarveout = std::stoi(v);
        else if (k == "sprobe") t.smemProbe = std::stoi(v);
        else if (k == "bbs") t.buildBlockSize = std::stoi(v);
        else if (k == "bvec") t.buildVectorRows = std::stoi(v);
        else if (k == "htf") t.hashFill = std::stoi(v);
        else if (k == "warm") t.warmLog2 = std::stoi(v);
        else if (k == "wprobe") t.warmProbe = std::stoi(v);
        else if (k == "tkb") t.topkBlocks = std::stoi(v);
        else throw std::runtime_error("tune: unknown key '" + k + "'");
    }
    if (t.blockSize < 32 || t.blockSize > 1024 || t.blockSize % 32)
        throw std::runtime_error("tune: bs must be a multiple of 32 in [32,1024]");
    if (t.scan.tileRows < 0 || t.scan.tileRows % 16) throw std::runtime_error("tune: tile must be a multiple of 16 (0 = auto)");
    if (t.scan.prefetchRows < 0 || t.scan.prefetchRows > 16) throw std::runtime_error("tune: pf must be in [0,16]");
    if (t.smemCarveout < -1 || t.smemCarveout > 100) throw std::runtime_error("tune: carve must be -1 or in [0,100]");
    if (t.hashFill < 100 || t.hashFill > 800) throw std::runtime_error("tune: htf must be in [100,800] (percent)");
    if (t.warmLog2 != 0 && (t.warmLog2 < 8 || t.warmLog2 > 22))
        throw std::runtime_error("tune: warm must be 0 or in [8,22] (log2 of the warm table's slots)");
    if (t.warmProbe < 1 || t.warmProbe > 64) throw std::runtime_error("tune: wprobe must be in [1,64]");
    if (t.topkBlocks < 1 || t.topkBlocks > 1184) throw std::runtime_error("tune: tkb must be in [1,1184]");
    if (t.buildBlockSize != 0 && (t.buildBlockSize < 64 || t.buildBlockSize > 1024 || t.buildBlockSize % 32))
        throw std::runtime_error("tune: bbs must be 0 or a multiple of 32 in [64,1024]");
    return t;
}

// ===================================================================
// Builders
// ===================================================================
namespace {

struct Spec {
    SpecMap m;
    std::set<std::string> used;
    std::string str(const std::string& k, const std::string& def) {
        used.insert(k);
        auto it = m.find(k);
        return it == m.end() ? def : it->second;
    }
    long long num(const std::string& k, long long def) {
        used.insert(k);
        auto it = m.find(k);
        if (it == m.end()) return def;
        size_t p = 0;
        long long v = std::stoll(it->second, &p);
        if (p != it->second.size()) throw std::runtime_error("spec: '" + k + "' is not an integer");
        return v;
    }
    bool has(const std::string& k) const { return m.count(k) != 0; }
    void finish() {
        for (const auto& [k, v] : m)
            if (!used.count(k)) throw std::runtime_error("spec: unknown key '" + k + "' for this template");
    }
};

std::string L(long long v) { return std::to_string(v) + "ll"; }

// Slots requested for a hash table of `groups` expected groups.
std::string hashCapacity(const std::string& groups, const TuneConfig& tune) {
    if (tune.hashFill == 200) return "2 * (" + groups + ")";
    return "(" + groups + ") * " + std::to_string(tune.hashFill) + " / 100";
}

// `late` names columns read only by rows that survive a selective operator
// (semi-join / hash probe); with late materialisation they are not staged.
std::unique_ptr<CudaGridStrideScan> makeScan(CudaQueryPlan& plan, const std::string& table,
                                             const std::vector<std::string>& cols, const TuneConfig& tune,
                                             bool allowTma = true, const std::vector<std::string>& late = {}) {
    const TableDef& td = catalogTable(table);
    auto scan = std::make_unique<CudaGridStrideScan>(table, "row", "i");
    for (const auto& c : cols) scan->addColumn(c, td.col(c).cudaType);
    for (const auto& c : late) scan->addColumn(c, td.col(c).cudaType, tune.lateMaterialize);
    ScanConfig sc = tune.scan;
    if (!allowTma) sc.mode = ScanConfig::Direct;
    scan->setConfig(sc);
    bool seen = false;
    for (const auto& t : plan.tables) seen |= (t == table);
    if (!seen) plan.tables.push_back(table);
    return scan;
}

CudaQueryPlan::Phase& appendPhase(CudaQueryPlan& plan, const std::string& name, std::unique_ptr<CudaOperator> root,
                                  const TuneConfig& tune) {
    CudaQueryPlan::Phase ph;
    ph.name = name;
    ph.root = std::move(root);
    ph.threadgroupSize = tune.blockSize;
    ph.minBlocksPerSM = std::max(1, std::min(tune.minBlocksPerSM, 2048 / tune.blockSize));
    ph.smemCarveout = tune.smemCarveout;
    plan.phases.push_back(std::move(ph));
    return plan.phases.back();
}

// ---- q1: scan -> filter -> few-group aggregate (reference buildQ1Plan,
// metal_plan_builder.cpp:309-354). Buckets follow the reference's order:
// (flag_a=='A'?0 : flag_a=='N'?2 : 4) + (flag_b=='F'?0:1).
CudaQueryPlan buildQ1(Spec& s, const TuneConfig& tune) {
    CudaQueryPlan plan;
    plan.name = "Q1";
    const long long shipLe = s.num("ship_le", 2436);
    const std::string i = "i";
    auto scan = makeScan(plan, "fact",
                         {"f_ship_day", "f_quantity", "f_price", "f_discount", "f_tax", "f_flag_a", "f_flag_b"}, tune);
    auto filtered = std::make_unique<CudaSelection>(std::move(scan), "f_ship_day[i] <= " + std::to_string(shipLe));
    const std::string bucket =
        "((f_flag_a[i] == 'A' ? 0 : (f_flag_a[i] == 'N' ? 2 : 4)) + (f_flag_b[i] == 'F' ? 0 : 1))";
    auto agg = std::make_unique<CudaKeyedAgg>(std::move(filtered), "d_q1_aggs", bucket, 6, 7, "42");
    agg->addAggregate("sum_qty", 0, "f_quantity[i]", "add", false);
    agg->addAggregate("sum_base_price", 1, "f_price[i]", "add", false);
    agg->addAggregate("sum_disc_price", 2, "f_price[i] * (100ll - f_discount[i])", "add", false);
    agg->addAggregate("sum_charge", 3, "f_price[i] * (100ll - f_discount[i]) * (100ll + f_tax[i])", "add", true);
    agg->addAggregate("sum_disc", 5, "f_discount[i]", "add", false);
    agg->addAggregate("count_order", 6, "1", "add", false);
    if (tune.keyedStrategy) agg->setStrategy((CudaKeyedAgg::Strategy)tune.keyedStrategy);
    appendPhase(plan, "Q1_reduce", std::move(agg), tune);
    plan.chunkable = true;
    plan.decorate.push_back([](CudaResultSchema& rs) {
        rs.keyedAgg.keys = {{"flag_a", 2, 3, {"A", "N", "R"}}, {"flag_b", 1, 2, {"F", "O"}}};
        rs.keyedAgg.derived = {{"avg_qty", "sum_qty", "count_order"},
                               {"avg_price", "sum_base_price", "count_order"},
                               {"avg_disc", "sum_disc", "count_order"}};
    });
    return plan;
}

// ---- q6: scan -> filter -> scalar sum (reference buildQ6Plan,
// metal_plan_builder.cpp:253-303).
CudaQueryPlan buildQ6(Spec& s, const TuneConfig& tune) {
    CudaQueryPlan plan;
    plan.name = "Q6";
    const long long ge = s.num("ship_ge", 365), lt = s.num("ship_lt", 730);
    const long long dlo = s.num("disc_lo", 5), dhi = s.num("disc_hi", 7), qlt = s.num("qty_lt", 24);
    auto scan = makeScan(plan, "fact", {"f_ship_day", "f_quantity", "f_price", "f_discount"}, tune);
    const std::string pred = "(f_ship_day[i] >= " + std::to_string(ge) + " && f_ship_day[i] < " + std::to_string(lt) +
                             ") && (f_discount[i] >= " + L(dlo) + " && f_discount[i] <= " + L(dhi) +
                             ") && (f_quantity[i] < " + L(qlt) + ")";
    auto filtered = std::make_unique<CudaSelection>(std::move(scan), pred);
    auto reduce = std::make_unique<CudaTGReduce>(std::move(filtered), "d_q6");
    reduce->addAccumulator("revenue", "f_price[i] * f_discount[i]", "wide");
    reduce->setResultAlias("revenue", 0);
    appendPhase(plan, "Q6_reduce", std::move(reduce), tune);
    plan.chunkable = true;
    return plan;
}

// ---- semi-join + group-by (+ top-k): the join's parts as kernel source over the dim / probe columns: the
// build-side and probe-side filters, the summed expression, the group
// count when the caller supplies it (groups < 0: sized on the device, or
// by the build's distinct count in the unsplit plan), and k (0 = every
// group, no top-k).
struct JoinAggParts {
    std::string buildPred, probePred, revenue;
    long long k = 10;
    long long groups = -1;
};

CudaQueryPlan buildJoinAgg(const JoinAggParts& jp, const TuneConfig& tune) {
    CudaQueryPlan plan;
    plan.name = jp.k > 0 ? "JOIN_TOPK" : "JOIN_GROUPS";
    const long long k = jp.k;
    const bool given = jp.groups >= 0;
    const long long groups = jp.groups;
    auto filtered = [](std::unique_ptr<CudaOperator> in, const std::string& pred) -> std::unique_ptr<CudaOperator> {
        if (pred.empty()) return in;
        return std::make_unique<CudaSelection>(std::move(in), pred);
    };
    const TuneConfig splitTune = [&] {
        TuneConfig t = tune;
        // every group: the host-sized plan, whose table is filled whole, so
        // the collector can read every slot (the device-sized table only
        // initialises the slots it uses)
        if (k <= 0) t.splitJoin = false;
        // the split plan's build and probe consumers set bits and look them
        // up per row: their automatic tiles hold whole consumer rounds
        if (t.splitJoin) t.scan.wholeRounds = true;
        return t;
    }();
    {
        const TuneConfig bt = splitTune.forBuild();
        auto scan = makeScan(plan, "dim", {"b_key", "b_order_day", "b_segment"}, bt);
        auto f = filtered(std::move(scan), jp.buildPred);
        auto bm = std::make_unique<CudaBitmapBuild>(std::move(f), "jb_bitmap", "b_key[i]", "max_b_key / 32 + 1");
        // the split plan counts the bitmap's keys after the build (in its
        // probe), so the build sets bits without waiting on their old values
        if (!splitTune.splitJoin) bm->setDistinctCounter("jb_distinct");
        appendPhase(plan, "JT_build", std::move(bm), bt);
    }
    const std::string cap = "2 * max(jt_groups, 1)";
    if (splitTune.splitJoin) {
        // The probe only lists the matched rows; a second phase gathers
        // their price / discount and aggregates. A matched row's slow work
        // (gathers, hash insert) then never holds a staged tile, and the
        // group table is sized by min(qualifying build keys, matched rows).
        {
            auto scan = makeScan(plan, "probe", {"p_fk", "p_ship_day"}, splitTune);
            auto f = filtered(std::move(scan), jp.probePred);
            auto pr = std::make_unique<CudaBitmapProbe>(std::move(f), "jb_bitmap", "p_fk[i]");
            pr->setPopcountInto("jb_distinct");
            auto mt = std::make_unique<CudaMaterialize>(std::move(pr), "jm_n", "n_probe");
            mt->addColumn("jm_rows", "unsigned", "(unsigned)_row");
            mt->addColumn("jm_fk", "int", "p_fk[i]");  // the group key rides along: no gather of it later
            mt->setIntermediate(true);
            appendPhase(plan, "JT_probe", std::move(mt), splitTune);
        }
        // No host round trip sizes the group table: it is allocated for
        // min(probe rows, build keys) groups and JT_init / JT_group derive
        // its slot count on the device from the two counters.
        // every thread reads the two counters: through L1 (written by
        // earlier kernels), not as one L2 line hammered by all warps
        const std::string devGroups = "min(__ldg(jm_n), __ldg(jb_distinct))";
        const std::string bound = "2 * max(min(n_probe, max_b_key + 1), 1)";
        const std::vector<std::string> counters = {"jm_n", "jb_distinct"};
        appendPhase(plan, "JT_init",
                    std::make_unique<CudaHashInit>("jg", "int", HashLayout::Linear, std::vector<std::string>{"revenue"},
                                                   devGroups, bound, counters),
                    splitTune);
        {
            auto ls = std::make_unique<CudaSlotListScan>("jm_rows", "jm_n");
            ls->addListColumn("jm_fk", "int", "_jm_fk");
            ls->addGatherColumn("p_price", "long long", "probe");
            ls->addGatherColumn("p_discount", "long long", "probe");
            auto gb = std::make_unique<CudaHashGroupBy>(std::move(ls), "jg", "_jm_fk", "int", cap, HashLayout::Linear,
                                                        splitTune.maxProbe);
            gb->addAggregate("revenue", jp.revenue);
            gb->setWarpAggregate(splitTune.warpAggregate);
            gb->setSlotList(true);
            gb->setDeviceCapacity(devGroups, bound, counters);
            appendPhase(plan, "JT_group", std::move(gb), splitTune);
        }
    } else {
        auto scan = makeScan(plan, "probe", {"p_fk", "p_ship_day"}, splitTune, true, {"p_price", "p_discount"});
        auto f = filtered(std::move(scan), jp.probePred);
        auto pr = std::make_unique<CudaBitmapProbe>(std::move(f), "jb_bitmap", "p_fk[i]");
        auto gb = std::make_unique<CudaHashGroupBy>(std::move(pr), "jg", "p_fk[i]", "int", cap, HashLayout::Linear,
                                                    splitTune.maxProbe);
        gb->addAggregate("revenue", jp.revenue);
        gb->setWarpAggregate(splitTune.warpAggregate);
        gb->setSlotList(true);
        appendPhase(plan, "JT_probe_group", std::move(gb), splitTune);
    }
    if (k > 0) {
        // only the slots whose groups were created (the probe's slot list)
        auto lscan = std::make_unique<CudaSlotListScan>("jg_slotlist", "jg_nslots");
        auto tk = std::make_unique<CudaTopK>(std::move(lscan), "jt_top", "(long long)(int)jg_keys[i]",
                                             "(long long)jg_revenue[i]", (int)k, splitTune.topkBlocks);
        auto& ph = appendPhase(plan, "JT_topk", std::move(tk), splitTune);
        ph.minBlocksPerSM = 1;  // the register-resident top-k lists must not be capped by an occupancy hint
        ph.extraBuffers.push_back({"jg_keys", "unsigned", true, false});
        ph.extraBuffers.push_back({"jg_revenue", "unsigned long long", true, false});
    }
    if (!splitTune.splitJoin) {
        CudaQueryPlan::SizingStep st;
        st.symbol = "jt_groups";
        st.afterPhase = 1;
        if (given) st.fallbackExpr = std::to_string(groups);
        else st.counterBuffer = "jb_distinct";
        plan.sizing.push_back(st);
    }
    if (k > 0) {
        plan.decorate.push_back([](CudaResultSchema& rs) {
            rs.topk.keyName = "key";
            rs.topk.valueName = "revenue";
        });
        plan.cpuSort = CudaQueryPlan::CpuSort{{{"revenue", true}, {"key", false}}, (int)k};
    } else {
        plan.decorate.push_back([](CudaResultSchema& rs) { rs.hashAgg.keyName = "key"; });
    }
    return plan;
}

// ---- join_topk: bitmap semi-join build -> probe + hash group-by ->
// top-k (reference Q3 shape: metal_plan_builder.cpp:1170-1239 + host top-k
// codegen_main.cpp:1211-1248). The build's distinct counter is the exact
// sizing pass for the group table; `groups=N` supplies it instead.
CudaQueryPlan buildJoinTopK(Spec& s, const TuneConfig& tune) {
    const long long seg = s.num("seg", 1), odLt = s.num("od_lt", 1170), shipGt = s.num("ship_gt", 1170);
    JoinAggParts jp;
    jp.buildPred = "b_segment[i] == " + std::to_string(seg) + " && b_order_day[i] < " + std::to_string(odLt);
    jp.probePred = "p_ship_day[i] > " + std::to_string(shipGt);
    jp.revenue = "p_price[i] * (100ll - p_discount[i])";
    jp.k = s.num("k", 10);
    if (jp.k < 1) throw std::runtime_error("join_topk: k must be at least 1");
    if (s.has("groups")) jp.groups = s.num("groups", 0);
    return buildJoinAgg(jp, tune);
}

// ---- join_rows: the Q3 semi-join with its matching probe rows
// materialised (row id, key, revenue) instead of aggregated — the
// reference's Materialize operator (metal_operators.cpp:618-643) on the
// join of metal_plan_builder.cpp:1170-1239. Rows come out in no order, as
// the reference's atomic output positions do; the capacity is the probe
// table (every row may match).
CudaQueryPlan buildJoinRows(Spec& s, const TuneConfig& tune) {
    CudaQueryPlan plan;
    plan.name = "JOIN_ROWS";
    const long long seg = s.num("seg", 1), odLt = s.num("od_lt", 1170), shipGt = s.num("ship_gt", 1170);
    {
        auto scan = makeScan(plan, "dim", {"b_key", "b_order_day", "b_segment"}, tune);
        auto f = std::make_unique<CudaSelection>(std::move(scan), "b_segment[i] == " + std::to_string(seg) +
                                                                      " && b_order_day[i] < " + std::to_string(odLt));
        auto bm = std::make_unique<CudaBitmapBuild>(std::move(f), "jb_bitmap", "b_key[i]", "max_b_key / 32 + 1");
        appendPhase(plan, "JR_build", std::move(bm), tune);
    }
    {
        auto scan = makeScan(plan, "probe", {"p_fk", "p_ship_day"}, tune, true, {"p_price", "p_discount"});
        auto f = std::make_unique<CudaSelection>(std::move(scan), "p_ship_day[i] > " + std::to_string(shipGt));
        auto pr = std::make_unique<CudaBitmapProbe>(std::move(f), "jb_bitmap", "p_fk[i]");
        auto mt = std::make_unique<CudaMaterialize>(std::move(pr), "jr_n", "n_probe");
        mt->addColumn("jr_row", "long long", "_row", "row");
        mt->addColumn("jr_key", "int", "p_fk[i]", "key");
        mt->addColumn("jr_revenue", "long long", "p_price[i] * (100ll - p_discount[i])", "revenue");
        appendPhase(plan, "JR_probe", std::move(mt), tune);
    }
    return plan;
}

// ---- join_direct: the reference's Q3 operator chain on the join tables
// (metal_plan_builder.cpp:1170-1239): the qualifying build rows fill two
// direct-address maps indexed by key (ArrayStore x2, sentinel -1), the
// probe looks its key up in the first (ArrayLookup) and adds its revenue
// into a dense per-key array (AtomicAgg); the reference's host post-step
// (top 10 of the dense array with the maps' attributes, codegen_main.cpp:
// 1211-1248) runs on the GPU: a top-k over the non-zero entries, then a
// gather of the top keys' map values.
CudaQueryPlan buildJoinDirect(Spec& s, const TuneConfig& tune) {
    CudaQueryPlan plan;
    plan.name = "JOIN_DIRECT";
    const long long seg = s.num("seg", 1), odLt = s.num("od_lt", 1170), shipGt = s.num("ship_gt", 1170);
    const long long k = s.num("k", 10);
    const std::string keys = "max_b_key + 1";
    {
        auto scan = makeScan(plan, "dim", {"b_key", "b_order_day", "b_segment"}, tune);
        auto f = std::make_unique<CudaSelection>(std::move(scan), "b_segment[i] == " + std::to_string(seg) +
                                                                      " && b_order_day[i] < " + std::to_string(odLt));
        auto day = std::make_unique<CudaArrayStore>(std::move(f), "jd_day", "b_key[i]", "b_order_day[i]", "int", keys);
        auto sg = std::make_unique<CudaArrayStore>(std::move(day), "jd_seg", "b_key[i]", "(int)b_segment[i]", "int", keys);
        appendPhase(plan, "JD_build", std::move(sg), tune);
    }
    {
        auto scan = makeScan(plan, "probe", {"p_fk", "p_ship_day"}, tune, true, {"p_price", "p_discount"});
        auto f = std::make_unique<CudaSelection>(std::move(scan), "p_ship_day[i] > " + std::to_string(shipGt));
        auto lk = std::make_unique<CudaArrayLookup>(std::move(f), "jd_day", "p_fk[i]", "_oday", "int", -1);
        auto ag = std::make_unique<CudaAtomicAgg>(std::move(lk), "jd_rev", "p_fk[i]",
                                                  "p_price[i] * (100ll - p_discount[i])", keys);
        appendPhase(plan, "JD_probe", std::move(ag), tune);
    }
    {
        auto sc = std::make_unique<CudaBufferScan>("n_jd", keys, "i");
        auto nz = std::make_unique<CudaSelection>(std::move(sc), "jd_rev[i] != 0ull");
        auto tk = std::make_unique<CudaTopK>(std::move(nz), "jd_top", "i", "(long long)jd_rev[i]", (int)k);
        auto& ph = appendPhase(plan, "JD_topk", std::move(tk), tune);
        ph.minBlocksPerSM = 1;  // the register-resident top-k lists must not be capped by an occupancy hint
        ph.extraBuffers.push_back({"jd_rev", "unsigned long long", true, false});
    }
    {
        auto g = std::make_unique<CudaIndexGather>("jd_top_keys", "jd_top_count", (int)k);
        g->addColumn("jd_day", "int", "jd_top_day", "order_day");
        g->addColumn("jd_seg", "int", "jd_top_seg", "segment");
        auto& ph = appendPhase(plan, "JD_attrs", std::move(g), tune);
        ph.threadgroupSize = 32;
        ph.minBlocksPerSM = 1;
    }
    plan.decorate.push_back([](CudaResultSchema& rs) {
        rs.kind = CudaResultSchema::TOPK;
        rs.topk.keyName = "key";
        rs.topk.valueName = "revenue";
    });
    plan.cpuSort = CudaQueryPlan::CpuSort{{{"revenue", true}, {"key", false}}, (int)k};
    return plan;
}

// ---- anti_join: the reference's Q22 operator chain (metal_plan_builder.cpp:
// 1304-1357) on the join tables: a bitmap of the qualifying build keys, then
// the probe rows whose key is NOT in it (AntiBitmapProbe), binned by a
// computed expression (ComputeExpr: the discount) and aggregated per bin by
// AtomicCount (rows) and AtomicAgg (sum of price).
CudaQueryPlan buildAntiJoin(Spec& s, const TuneConfig& tune) {
    CudaQueryPlan plan;
    plan.name = "ANTI_JOIN";
    const long long seg = s.num("seg", 1), odLt = s.num("od_lt", 1170), shipGt = s.num("ship_gt", 1170);
    const std::string bins = "11";  // discount 0..10 (hundredths)
    {
        auto scan = makeScan(plan, "dim", {"b_key", "b_order_day", "b_segment"}, tune);
        auto f = std::make_unique<CudaSelection>(std::move(scan), "b_segment[i] == " + std::to_string(seg) +
                                                                      " && b_order_day[i] < " + std::to_string(odLt));
        auto bm = std::make_unique<CudaBitmapBuild>(std::move(f), "aj_bitmap", "b_key[i]", "max_b_key / 32 + 1");
        appendPhase(plan, "AJ_build", std::move(bm), tune);
    }
    {
        auto scan = makeScan(plan, "probe", {"p_fk", "p_ship_day", "p_discount"}, tune, true, {"p_price"});
        auto f = std::make_unique<CudaSelection>(std::move(scan), "p_ship_day[i] > " + std::to_string(shipGt));
        auto anti = std::make_unique<CudaAntiBitmapProbe>(std::move(f), "aj_bitmap", "p_fk[i]");
        auto bin = std::make_unique<CudaComputeExpr>(std::move(anti), "_bin", "int", "(int)p_discount[i]");
        auto cnt = std::make_unique<CudaAtomicCount>(std::move(bin), "aj_count", "_bin", bins);
        auto sum = std::make_unique<CudaAtomicAgg>(std::move(cnt), "aj_sum", "_bin", "p_price[i]", bins);
        sum->setWarpAggregate(true);
        sum->setSharedCache(4, 4);
        appendPhase(plan, "AJ_probe", std::move(sum), tune);
    }
    plan.decorate.push_back([bins](CudaResultSchema& rs) {
        rs.kind = CudaResultSchema::DIRECT_AGG;
        rs.directAgg.sizeExpr = bins;
        rs.directAgg.keyName = "discount";
        rs.directAgg.aggs = {{"count", "aj_count"}, {"sum_price", "aj_sum"}};
    });
    return plan;
}

// ---- histogram: the reference's Q13 operator chain (metal_plan_builder.cpp:
// 1244-1299): AtomicCount of the filtered probe rows per build key, then
// for every build row an ArrayLookup of its key's count and an AtomicCount
// histogram over those counts (bin = rows per key, value = keys).
CudaQueryPlan buildHistogram(Spec& s, const TuneConfig& tune) {
    CudaQueryPlan plan;
    plan.name = "HISTOGRAM";
    const long long shipGt = s.num("ship_gt", 1170);
    const long long bins = s.num("bins", 256);
    if (bins < 1 || bins > 8192) throw std::runtime_error("histogram: bins must be in [1, 8192]");
    {
        auto scan = makeScan(plan, "probe", {"p_fk", "p_ship_day"}, tune);
        auto f = std::make_unique<CudaSelection>(std::move(scan), "p_ship_day[i] > " + std::to_string(shipGt));
        auto cnt = std::make_unique<CudaAtomicCount>(std::move(f), "h_count", "p_fk[i]", "max_b_key + 1");
        appendPhase(plan, "H_count", std::move(cnt), tune);
    }
    {
        auto scan = makeScan(plan, "dim", {"b_key"}, tune);
        auto lk = std::make_unique<CudaArrayLookup>(std::move(scan), "h_count", "b_key[i]", "_cnt", "long long", -1);
        auto hist = std::make_unique<CudaAtomicCount>(std::move(lk), "h_hist", "_cnt", std::to_string(bins));
        appendPhase(plan, "H_hist", std::move(hist), tune);
    }
    plan.decorate.push_back([bins](CudaResultSchema& rs) {
        rs.kind = CudaResultSchema::DIRECT_AGG;
        rs.directAgg.sizeExpr = std::to_string(bins);
        rs.directAgg.keyName = "rows_per_key";
        rs.directAgg.aggs = {{"keys", "h_hist"}};
    });
    return plan;
}

// ---- q6_selvec: the predicate variant in two phases over a selection
// bitmap: the first evaluates the predicate on its three columns and
// writes one bit per row (warp-ORed words); the second visits only the set
// bits and gathers price and discount of those rows for the sum.
CudaQueryPlan buildQ6SelVec(Spec& s, const TuneConfig& tune) {
    CudaQueryPlan plan;
    plan.name = "Q6_SELVEC";
    const long long ge = s.num("ship_ge", 365), lt = s.num("ship_lt", 730);
    const long long dlo = s.num("disc_lo", 5), dhi = s.num("disc_hi", 7), qlt = s.num("qty_lt", 24);
    {
        auto scan = makeScan(plan, "fact", {"f_ship_day", "f_quantity", "f_discount"}, tune);
        const std::string pred = "(f_ship_day[i] >= " + std::to_string(ge) + " && f_ship_day[i] < " + std::to_string(lt) +
                                 ") && (f_discount[i] >= " + L(dlo) + " && f_discount[i] <= " + L(dhi) +
                                 ") && (f_quantity[i] < " + L(qlt) + ")";
        auto sel = std::make_unique<CudaSelection>(std::move(scan), pred);
        sel->setBitmapOut("q6_sel", "n_fact");
        appendPhase(plan, "Q6S_select", std::move(sel), tune);
    }
    {
        auto ss = std::make_unique<CudaSelectionScan>("fact", "q6_sel");
        ss->addColumn("f_price", "long long");
        ss->addColumn("f_discount", "long long");
        auto reduce = std::make_unique<CudaTGReduce>(std::move(ss), "d_q6s");
        reduce->addAccumulator("revenue", "f_price[i] * f_discount[i]", "wide");
        reduce->setResultAlias("revenue", 0);
        appendPhase(plan, "Q6S_sum", std::move(reduce), tune);
    }
    return plan;
}

// ---- multi_join: the reference's Q5 plan shape (metal_plan_builder.cpp:
// 894-1015), five phases over the snowflake: a bitmap of the region's
// nations; customer and supplier nation maps of those nations (BitmapProbe
// -> ArrayStore); the date-filtered orders' customer nation (ArrayLookup ->
// ArrayStore); then every line looks up its order's and its supplier's
// nation, keeps the lines whose two nations agree (Selection) and adds its
// revenue per nation (AtomicAgg, 25 bins).
CudaQueryPlan buildMultiJoin(Spec& s, const TuneConfig& tune) {
    CudaQueryPlan plan;
    plan.name = "MULTI_JOIN";
    const long long region = s.num("region", 2), dayGe = s.num("day_ge", 730), dayLt = s.num("day_lt", 1095);
    {
        auto scan = makeScan(plan, "nation", {"n_key", "n_region"}, tune, false);
        auto f = std::make_unique<CudaSelection>(std::move(scan), "n_region[i] == " + std::to_string(region));
        auto bm = std::make_unique<CudaBitmapBuild>(std::move(f), "mj_nations", "n_key[i]", "1");
        auto& ph = appendPhase(plan, "MJ_nations", std::move(bm), tune);
        ph.threadgroupSize = 32;
    }
    {
        auto scan = makeScan(plan, "cust", {"c_key", "c_nation"}, tune);
        auto pr = std::make_unique<CudaBitmapProbe>(std::move(scan), "mj_nations", "c_nation[i]");
        auto st = std::make_unique<CudaArrayStore>(std::move(pr), "mj_cust_nation", "c_key[i]", "c_nation[i]", "int",
                                                   "max_c_key + 1");
        appendPhase(plan, "MJ_cust", std::move(st), tune);
    }
    {
        auto scan = makeScan(plan, "supp", {"s_key", "s_nation"}, tune);
        auto pr = std::make_unique<CudaBitmapProbe>(std::move(scan), "mj_nations", "s_nation[i]");
        auto st = std::make_unique<CudaArrayStore>(std::move(pr), "mj_supp_nation", "s_key[i]", "s_nation[i]", "int",
                                                   "max_s_key + 1");
        appendPhase(plan, "MJ_supp", std::move(st), tune);
    }
    {
        auto scan = makeScan(plan, "ord", {"o_key", "o_cust", "o_day"}, tune);
        auto f = std::make_unique<CudaSelection>(std::move(scan), "o_day[i] >= " + std::to_string(dayGe) +
                                                                      " && o_day[i] < " + std::to_string(dayLt));
        auto lk = std::make_unique<CudaArrayLookup>(std::move(f), "mj_cust_nation", "o_cust[i]", "_cn", "int", -1);
        auto st = std::make_unique<CudaArrayStore>(std::move(lk), "mj_ord_nation", "o_key[i]", "_cn", "int",
                                                   "max_o_key + 1");
        appendPhase(plan, "MJ_orders", std::move(st), tune);
    }
    {
        auto scan = makeScan(plan, "line", {"l_okey", "l_supp"}, tune, true, {"l_price", "l_discount"});
        auto lo = std::make_unique<CudaArrayLookup>(std::move(scan), "mj_ord_nation", "l_okey[i]", "_cn", "int", -1);
        auto ls = std::make_unique<CudaArrayLookup>(std::move(lo), "mj_supp_nation", "l_supp[i]", "_sn", "int", -1);
        auto same = std::make_unique<CudaSelection>(std::move(ls), "_cn == _sn");
        auto ag = std::make_unique<CudaAtomicAgg>(std::move(same), "mj_revenue", "_cn",
                                                  "l_price[i] * (100ll - l_discount[i])", "25");
        ag->setWarpAggregate(true);
        ag->setSharedCache(5, 2);
        appendPhase(plan, "MJ_lines", std::move(ag), tune);
    }
    plan.decorate.push_back([](CudaResultSchema& rs) {
        rs.kind = CudaResultSchema::DIRECT_AGG;
        rs.directAgg.sizeExpr = "25";
        rs.directAgg.keyName = "nation";
        rs.directAgg.aggs = {{"revenue", "mj_revenue"}};
    });
    return plan;
}

// ---- groupby: high-cardinality hash group-by, count + sum (reference
// Q18 shape metal_plan_builder.cpp:1529-1545, which aggregates into a
// direct-address array; here an open-addressing table keyed by int64).
CudaQueryPlan buildGroupBy(Spec& s, const TuneConfig& tune) {
    CudaQueryPlan plan;
    plan.name = "GROUPBY";
    const std::string groupsExpr = s.str("groups", "zgroups");
    auto scan = makeScan(plan, "zprobe", {"z_key", "z_value"}, tune);
    auto gb = std::make_unique<CudaHashGroupBy>(std::move(scan), "zg", "z_key[i]", "long long",
                                                hashCapacity(groupsExpr, tune), tune.hashLayout, tune.maxProbe);
    gb->addAggregate("count", "1");
    gb->addAggregate("sum", "z_value[i]");
    gb->setWarpAggregate(tune.warpAggregate);
    gb->setSharedPreAgg(tune.smemPreAggLog2, tune.smemProbe);
    if (tune.warmLog2) gb->setWarmTier(tune.warmLog2, tune.warmProbe);
    appendPhase(plan, "GB_aggregate", std::move(gb), tune);
    if (tune.warmLog2)
        appendPhase(plan, "GB_warm_flush",
                    std::make_unique<CudaHashWarmFlush>("zg", hashCapacity(groupsExpr, tune), tune.hashLayout,
                                                        tune.maxProbe, std::vector<std::string>{"count", "sum"},
                                                        tune.warmLog2, false),
                    tune);
    return plan;
}

// ---- groupby_sorted: the skewed-key group-by with every group returned
// in ORDER BY sum DESC, key ASC — the reference sorts such group rows on
// the host (the Q18 post-processing, codegen_main.cpp:1105-1721); here the
// created groups are compacted and merge-sorted on the GPU. The plan
// carries merge passes for up to 2048 << 15 groups; passes beyond what the
// run's group count needs return at once.
CudaQueryPlan buildGroupBySorted(Spec& s, const TuneConfig& tune) {
    CudaQueryPlan plan;
    plan.name = "GROUPBY_SORTED";
    const std::string groupsExpr = s.str("groups", "zgroups");
    const int passes = (int)s.num("passes", 15);
    if (passes < 1 || passes > 20) throw std::runtime_error("groupby_sorted: passes must be in [1, 20]");
    {
        auto scan = makeScan(plan, "zprobe", {"z_key", "z_value"}, tune);
        auto gb = std::make_unique<CudaHashGroupBy>(std::move(scan), "gs", "z_key[i]", "long long",
                                                    hashCapacity(groupsExpr, tune), tune.hashLayout == HashLayout::Packed
                                                        ? HashLayout::Linear : tune.hashLayout, tune.maxProbe);
        gb->addAggregate("count", "1");
        gb->addAggregate("sum", "z_value[i]");
        gb->setWarpAggregate(tune.warpAggregate);
        gb->setSharedPreAgg(tune.smemPreAggLog2, tune.smemProbe);
        gb->setSlotList(true);
        appendPhase(plan, "GS_group", std::move(gb), tune);
    }
    const std::string cap = "max(" + groupsExpr + ", 1)";
    {
        auto ls = std::make_unique<CudaSlotListScan>("gs_slotlist", "gs_nslots");
        auto mt = std::make_unique<CudaMaterialize>(std::move(ls), "gsc_n", cap);
        mt->addColumn("gsc_key", "long long", "(long long)gs_keys[i]");
        mt->addColumn("gsc_count", "long long", "(long long)gs_count[i]");
        mt->addColumn("gsc_sum", "long long", "(long long)gs_sum[i]");
        mt->setIntermediate(true);
        auto& ph = appendPhase(plan, "GS_compact", std::move(mt), tune);
        ph.extraBuffers.push_back({"gs_keys", "unsigned long long", true, false});
        ph.extraBuffers.push_back({"gs_count", "unsigned long long", true, false});
        ph.extraBuffers.push_back({"gs_sum", "unsigned long long", true, false});
    }
    TuneConfig st = tune;
    st.blockSize = 512;
    st.minBlocksPerSM = 1;
    {
        auto sp = std::make_unique<CudaSortPass>(CudaSortPass::Mode::Chunks, "gss", "gsc_n", cap);
        sp->setInput("gsc_key", "gsc_count", "gsc_sum");
        appendPhase(plan, "GS_sort_chunks", std::move(sp), st);
    }
    for (int p = 0; p < passes; p++)
        appendPhase(plan, "GS_merge" + std::to_string(p),
                    std::make_unique<CudaSortPass>(CudaSortPass::Mode::Merge, "gss", "gsc_n", cap, p), st);
    {
        auto sp = std::make_unique<CudaSortPass>(CudaSortPass::Mode::Emit, "gss", "gsc_n", cap);
        sp->setOutputNames("key", "count", "sum");
        appendPhase(plan, "GS_emit", std::move(sp), st);
    }
    return plan;
}

// ---- hashjoin: GPU hash build (64-bit CAS) -> probe -> per-key sum of
// the build payload over matches (reference Q9/Q20 hash tables:
// query_preprocessing.cpp:352-386/443-479 built on the host, probed by
// metal_plan_builder.cpp:1598-1610/1968-1982).
CudaQueryPlan buildHashJoin(Spec& s, const TuneConfig& tune) {
    CudaQueryPlan plan;
    plan.name = "HASHJOIN";
    (void)s;
    const std::string cap = hashCapacity("n_zbuild", tune);
    {
        auto scan = makeScan(plan, "zbuild", {"zb_key", "zb_payload"}, tune);
        auto hb = std::make_unique<CudaHashBuild>(std::move(scan), "hj", "zb_key[i]", "long long", cap, tune.hashLayout,
                                                  tune.maxProbe);
        hb->addPayload("payload", "int", "zb_payload[i]");
        appendPhase(plan, "HJ_build", std::move(hb), tune);
    }
    // The summed column is the build key's own payload, so the sum per key
    // is payload × matches: the probe only counts matches per slot (one
    // random slot touch per probe row instead of payload, sum and count),
    // and a pass over the slots multiplies (eager aggregation).
    const std::string slots = hashSlotsExpr(cap);
    {
        auto scan = makeScan(plan, "zprobe", {"z_key"}, tune);
        auto pr = std::make_unique<CudaHashProbe>(std::move(scan), "hj", "z_key[i]", "long long", cap, "_slot",
                                                  tune.hashLayout, tune.maxProbe);
        auto ag = std::make_unique<CudaAtomicAgg>(std::move(pr), "hj_count", "_slot", "1ll", slots);
        ag->setWarpAggregate(tune.warpAggregate);
        ag->setSharedCache(tune.smemPreAggLog2, tune.smemProbe);
        auto& ph = appendPhase(plan, "HJ_probe_count", std::move(ag), tune);
        ph.extraBuffers.push_back({"hj_keys", "unsigned long long", true, false});
    }
    {
        auto sc = std::make_unique<CudaBufferScan>("n_hj_slots", slots, "s");
        auto st = std::make_unique<CudaArrayStore>(std::move(sc), "hj_sum", "s",
                                                   "(long long)hj_payload[s] * (long long)hj_count[s]", "long long", slots);
        st->setDense(true);
        auto& ph = appendPhase(plan, "HJ_sum", std::move(st), tune);
        ph.extraBuffers.push_back({"hj_payload", "int", true, false});
        ph.extraBuffers.push_back({"hj_count", "unsigned long long", true, false});
    }
    plan.decorate.push_back([cap](CudaResultSchema& rs) {
        rs.kind = CudaResultSchema::HASH_AGG;
        rs.hashAgg.keyBuffer = "hj_keys";
        rs.hashAgg.keyType = "unsigned long long";
        rs.hashAgg.capacitySymbol = hashSlotsExpr(cap);
        rs.hashAgg.aggs = {{"count", "hj_count"}, {"sum", "hj_sum"}};
    });
    return plan;
}

// ---- colmax: exact max of an integer column (the reference's max-key
// sizing pass, max_key_symbols.cpp:188-235, run on the GPU).
CudaQueryPlan buildColMax(Spec& s, const TuneConfig& tune) {
    CudaQueryPlan plan;
    const std::string table = s.str("table", "");
    const std::string col = s.str("col", "");
    plan.name = "COLMAX";
    auto scan = makeScan(plan, table, {col}, tune);
    // max over signed values as an unsigned max of (v ^ sign bit); the
    // zero fill of the output word is then the identity.
    auto r = std::make_unique<CudaTGReduce>(std::move(scan), "d_colmax");
    r->addAccumulator("max_biased", "(unsigned long long)(long long)" + col + "[i] ^ 0x8000000000000000ull", "umax");
    auto ag = std::move(r);
    appendPhase(plan, "COLMAX_" + col, std::move(ag), tune);
    return plan;
}

// ---- distinct: exact distinct count of (key % card) over rows passing a
// filter; the exact count pass of the mixed group-by templates.
// Constants of the mixed templates: compiled into the source, or (spec
// params=1) kernel arguments bound at launch from the registered symbols
// mix_thr / mix_card / mix_attr_lt, so one module serves every query of a
// template (a group key's remainder then goes through the invariant-divisor
// multiply-high, gpudb_mod_i32).
struct MixConsts {
    bool params = false;
    std::string thr, card, attrLt, keyMod;
    std::vector<CudaQueryPlan::Phase::SizeScalar> scalars;
    std::vector<std::string> prologue;
};

MixConsts mixConsts(Spec& s, const std::string& keyCol, bool grouped, bool join) {
    MixConsts c;
    c.params = s.num("params", 0) != 0;
    if (!c.params) {
        c.thr = std::to_string(s.num("thr", 10000));
        if (grouped) {
            c.card = L(s.num("card", 1024));
            c.keyMod = "(long long)" + keyCol + "[i] % " + c.card;
        }
        if (join) c.attrLt = std::to_string(s.num("attr_lt", 500));
        return c;
    }
    for (const char* k : {"thr", "card", "attr_lt"})
        if (s.has(k)) throw std::runtime_error(std::string("spec: '") + k + "' with params=1 (bound at launch from the symbol)");
    c.thr = "mix_thr";
    c.scalars.push_back({"mix_thr", "int", "mix_thr"});
    if (grouped) {
        c.card = "mix_card";
        c.scalars.push_back({"mix_card", "long long", "mix_card"});
        c.prologue.push_back("const gpudb_divmagic _mix_div = gpudb_divmagic_make(mix_card);");
        c.keyMod = "gpudb_mod_i32(" + keyCol + "[i], _mix_div)";
    }
    if (join) {
        c.attrLt = "mix_attr_lt";
        c.scalars.push_back({"mix_attr_lt", "int", "mix_attr_lt"});
    }
    return c;
}

void bindConsts(CudaQueryPlan::Phase& ph, const MixConsts& c) {
    for (const auto& x : c.scalars) ph.sizeScalars.push_back(x);
    for (const auto& l : c.prologue) ph.prologue.push_back(l);
}

CudaQueryPlan buildDistinct(Spec& s, const TuneConfig& tune) {
    CudaQueryPlan plan;
    plan.name = "DISTINCT";
    const std::string keyCol = s.str("key", "m_rank_u");
    const MixConsts mc = mixConsts(s, keyCol, true, false);
    const std::string bits = mc.params ? "mix_card / 32 + 1" : std::to_string(s.num("card", 1024) / 32 + 1);
    auto scan = makeScan(plan, "mix", {keyCol, "m_filter"}, tune);
    auto f = std::make_unique<CudaSelection>(std::move(scan), "m_filter[i] < " + mc.thr);
    auto bm = std::make_unique<CudaBitmapBuild>(std::move(f), "dc_bitmap", mc.keyMod, bits);
    bm->setDistinctCounter("dc_distinct");
    bindConsts(appendPhase(plan, "DC_count", std::move(bm), tune), mc);
    plan.decorate.push_back([](CudaResultSchema& rs) {
        rs.kind = CudaResultSchema::SCALAR_AGG;
        rs.scalarAggs = {{"distinct", "dc_distinct", false, 0}};
    });
    return plan;
}

// ---- mixed-workload templates (batched mixed-query form) ----------------
// mix_agg:     filter -> count + sum(value)
// mix_groupby: filter -> hash group-by on (rank % card): count + sum
// mix_topk:    mix_groupby -> top-k groups by sum
// mix_join:    bitmap semi-join on fk against mixdim(attr < a) -> count + sum
CudaQueryPlan buildMix(const std::string& tmpl, Spec& s, const TuneConfig& tune) {
    CudaQueryPlan plan;
    plan.name = tmpl;
    const bool grouped = tmpl == "mix_groupby" || tmpl == "mix_topk";
    const std::string keyCol = grouped ? s.str("key", "m_rank_u") : "m_rank_u";
    const MixConsts mc = mixConsts(s, keyCol, grouped, tmpl == "mix_join");
    const std::string filt = "m_filter[i] < " + mc.thr;
    if (tmpl == "mix_agg") {
        auto scan = makeScan(plan, "mix", {"m_filter", "m_value"}, tune);
        auto f = std::make_unique<CudaSelection>(std::move(scan), filt);
        auto r = std::make_unique<CudaTGReduce>(std::move(f), "d_mix");
        r->addAccumulator("count", "1", "long");
        r->addAccumulator("sum", "m_value[i]", "wide");
        bindConsts(appendPhase(plan, "MIX_agg", std::move(r), tune), mc);
        return plan;
    }
    if (tmpl == "mix_join") {
        {
            auto scan = makeScan(plan, "mixdim", {"md_key", "md_attr"}, tune);
            auto f = std::make_unique<CudaSelection>(std::move(scan), "md_attr[i] < " + mc.attrLt);
            auto bm = std::make_unique<CudaBitmapBuild>(std::move(f), "mj_bitmap", "md_key[i]", "max_md_key / 32 + 1");
            bindConsts(appendPhase(plan, "MIXJ_build", std::move(bm), tune), mc);
        }
        auto scan = makeScan(plan, "mix", {"m_fk", "m_filter"}, tune, true, {"m_value"});
        auto f = std::make_unique<CudaSelection>(std::move(scan), filt);
        auto pr = std::make_unique<CudaBitmapProbe>(std::move(f), "mj_bitmap", "m_fk[i]");
        auto r = std::make_unique<CudaTGReduce>(std::move(pr), "d_mixj");
        r->addAccumulator("count", "1", "long");
        r->addAccumulator("sum", "m_value[i]", "wide");
        bindConsts(appendPhase(plan, "MIXJ_probe", std::move(r), tune), mc);
        return plan;
    }
    const long long k = s.num("k", 10);
    const std::string groups = s.str("groups", "mix_groups");
    const std::string cap = "2 * max(" + groups + ", 1)";
    // compact=1: the created groups are gathered on the device into dense
    // (key, count, sum) arrays, so collecting the result copies groups x 24
    // bytes instead of the whole table
    const bool compact = tmpl == "mix_groupby" && s.num("compact", 0) != 0;
    auto scan = makeScan(plan, "mix", {keyCol, "m_filter", "m_value"}, tune);
    auto f = std::make_unique<CudaSelection>(std::move(scan), filt);
    auto gb = std::make_unique<CudaHashGroupBy>(std::move(f), "mg", mc.keyMod, "long long", cap, tune.hashLayout,
                                                tune.maxProbe);
    gb->addAggregate("count", "1");
    gb->addAggregate("sum", "m_value[i]");
    gb->setWarpAggregate(tune.warpAggregate);
    gb->setSharedPreAgg(tune.smemPreAggLog2, tune.smemProbe);
    gb->setSlotList(tmpl == "mix_topk" || compact);
    bindConsts(appendPhase(plan, "MIXG_group", std::move(gb), tune), mc);
    if (tmpl == "mix_topk") {
        auto lscan = std::make_unique<CudaSlotListScan>("mg_slotlist", "mg_nslots");
        auto tk = std::make_unique<CudaTopK>(std::move(lscan), "mt_top", "(long long)mg_keys[i]", "(long long)mg_sum[i]",
                                             (int)k);
        auto& ph = appendPhase(plan, "MIXG_topk", std::move(tk), tune);
        ph.minBlocksPerSM = 1;  // the register-resident top-k lists must not be capped by an occupancy hint
        ph.extraBuffers.push_back({"mg_keys", "unsigned long long", true, false});
        ph.extraBuffers.push_back({"mg_sum", "unsigned long long", true, false});
        plan.decorate.push_back([](CudaResultSchema& rs) { rs.topk.valueName = "sum"; });
    }
    if (compact) {
        auto lscan = std::make_unique<CudaSlotListScan>("mg_slotlist", "mg_nslots");
        auto mt = std::make_unique<CudaMaterialize>(std::move(lscan), "mgc_n", "max(" + groups + ", 1)");
        mt->addColumn("mgc_key", "long long", "(long long)mg_keys[i]", "key");
        mt->addColumn("mgc_count", "long long", "(long long)mg_count[i]", "count");
        mt->addColumn("mgc_sum", "long long", "(long long)mg_sum[i]", "sum");
        auto& ph = appendPhase(plan, "MIXG_compact", std::move(mt), tune);
        ph.minBlocksPerSM = 1;
        ph.extraBuffers.push_back({"mg_keys", "unsigned long long", true, false});
        ph.extraBuffers.push_back({"mg_count", "unsigned long long", true, false});
        ph.extraBuffers.push_back({"mg_sum", "unsigned long long", true, false});
    }
    return plan;
}

}  // namespace

std::vector<std::string> planTemplates() {
    return {"q1", "q6", "q6_selvec", "join_topk", "join_rows", "join_direct", "anti_join", "histogram", "multi_join", "groupby", "groupby_sorted",
            "hashjoin", "colmax", "distinct", "mix_agg", "mix_groupby", "mix_topk", "mix_join"};
}

CudaQueryPlan buildCudaPlan(const std::string& specStr, const TuneConfig& tune) {
    Spec s{parseSpec(specStr), {}};
    const std::string tmpl = s.str("template", "");
    CudaQueryPlan plan;
    if (tmpl == "q1" || tmpl == "scan_filter_groupagg") plan = buildQ1(s, tune);
    else if (tmpl == "q6" || tmpl == "scan_filter_sum") plan = buildQ6(s, tune);
    else if (tmpl == "join_topk") plan = buildJoinTopK(s, tune);
    else if (tmpl == "join_rows") plan = buildJoinRows(s, tune);
    else if (tmpl == "join_direct") plan = buildJoinDirect(s, tune);
    else if (tmpl == "anti_join") plan = buildAntiJoin(s, tune);
    else if (tmpl == "histogram") plan = buildHistogram(s, tune);
    else if (tmpl == "q6_selvec") plan = buildQ6SelVec(s, tune);
    else if (tmpl == "multi_join") plan = buildMultiJoin(s, tune);
    else if (tmpl == "groupby") plan = buildGroupBy(s, tune);
    else if (tmpl == "groupby_sorted") plan = buildGroupBySorted(s, tune);
    else if (tmpl == "hashjoin") plan = buildHashJoin(s, tune);
    else if (tmpl == "colmax") plan = buildColMax(s, tune);
    else if (tmpl == "distinct") plan = buildDistinct(s, tune);
    else if (tmpl == "mix_agg" || tmpl == "mix_groupby" || tmpl == "mix_topk" || tmpl == "mix_join")
        plan = buildMix(tmpl, s, tune);
    else throw std::runtime_error("buildCudaPlan: unknown template '" + tmpl + "'");
    s.finish();
    plan.spec = canonicalSpec(s.m);
    return plan;
}

// ===================================================================
// Planning from an analyzed query
// ===================================================================
namespace {

using namespace ir;

struct TableSplit {
    std::map<std::string, std::vector<PredPtr>> filters;  // engine table -> its filters
};

// The engine table a predicate's columns belong to ("" when it reads none).
std::string predicateTable(const PredPtr& p) {
    std::vector<ResolvedColumn> cols;
    collectColumns(p, cols);
    std::string t;
    for (const auto& c : cols) {
        if (!t.empty() && t != c.table)
            throw std::runtime_error("analyzed plan: a filter reads two tables (" + t + ", " + c.table +
                                     "); only equi-joins in the join clause connect tables");
        t = c.table;
    }
    return t;
}

bool isAliasRef(const ExprPtr& e, const std::string& alias) {
    if (!e || alias.empty()) return false;
    if (auto* c = std::get_if<ColRef>(&e->node)) return c->table.empty() && c->column == alias;
    return false;
}

std::optional<ResolvedColumn> plainColumn(const ExprPtr& e) {
    if (!e) return std::nullopt;
    if (auto* c = std::get_if<ColRef>(&e->node)) {
        try {
            return resolveColumn(c->table, c->column);
        } catch (const std::exception&) {
            return std::nullopt;
        }
    }
    return std::nullopt;
}

std::string aggName(AggFunc f) {
    switch (f) {
        case AggFunc::SUM: return "SUM";
        case AggFunc::COUNT: return "COUNT";
        case AggFunc::AVG: return "AVG";
        case AggFunc::MIN: return "MIN";
        case AggFunc::MAX: return "MAX";
        case AggFunc::COUNT_DISTINCT: return "COUNT(DISTINCT)";
    }
    return "?";
}

std::string aliasOf(const SelectTarget& t, size_t i) {
    if (!t.alias.empty()) return t.alias;
    if (t.agg && !t.agg->alias.empty()) return t.agg->alias;
    return "agg" + std::to_string(i);
}

std::unique_ptr<CudaOperator> scanFor(CudaQueryPlan& plan, const std::string& table,
                                      const std::vector<ResolvedColumn>& cols, const TuneConfig& tune) {
    std::vector<std::string> names;
    for (const auto& c : cols)
        if (c.table == table && std::find(names.begin(), names.end(), c.column) == names.end()) names.push_back(c.column);
    if (names.empty()) names.push_back(catalogTable(table).columns.front().name);  // COUNT(*) still scans
    return makeScan(plan, table, names, tune);
}

std::unique_ptr<CudaOperator> selectIf(std::unique_ptr<CudaOperator> in, const std::string& pred) {
    if (pred.empty()) return in;
    return std::make_unique<CudaSelection>(std::move(in), pred);
}

// One table, aggregates, no GROUP BY (the Q6 shape).
CudaQueryPlan planScalarAgg(const AnalyzedQuery& aq, const std::string& table, const std::string& name,
                            const TuneConfig& tune) {
    CudaQueryPlan plan;
    plan.name = name.empty() ? "SCALAR_AGG" : name;
    std::vector<ResolvedColumn> cols;
    for (const auto& f : aq.filters) collectColumns(f, cols);
    std::vector<std::tuple<std::string, std::string, std::string, int>> accs;  // alias, code, type, scale
    for (size_t i = 0; i < aq.targets.size(); i++) {
        const auto& t = aq.targets[i];
        if (!t.isAgg || !t.agg) throw std::runtime_error("analyzed plan: a non-aggregate target without GROUP BY");
        const auto& a = *t.agg;
        if (a.func == AggFunc::SUM) {
            collectColumns(a.innerExpr, cols);
            const Lowered v = exprToCuda(a.innerExpr, "i");
            accs.emplace_back(aliasOf(t, i), v.code, "wide", v.scale);
        } else if (a.func == AggFunc::COUNT) {
            accs.emplace_back(aliasOf(t, i), "1", "long", 0);
        } else {
            throw std::runtime_error("analyzed plan: " + aggName(a.func) + " in a scalar aggregate (SUM and COUNT "
                                     "are computed exactly on the device)");
        }
    }
    auto scan = scanFor(plan, table, cols, tune);
    auto f = selectIf(std::move(scan), combineFilters(aq.filters, "i"));
    auto r = std::make_unique<CudaTGReduce>(std::move(f), "d_ir");
    for (const auto& [alias, code, type, scale] : accs) {
        r->addAccumulator(alias, code, type);
        r->setResultAlias(alias, scale);
    }
    appendPhase(plan, plan.name + "_reduce", std::move(r), tune);
    plan.chunkable = true;
    return plan;
}

// One table, GROUP BY columns with known value sets (the Q1 shape).
CudaQueryPlan planKeyedAgg(const AnalyzedQuery& aq, const std::string& table, const std::vector<ResolvedColumn>& keys,
                           const std::vector<std::string>& keyNames, const std::string& name, const TuneConfig& tune) {
    CudaQueryPlan plan;
    plan.name = name.empty() ? "KEYED_AGG" : name;
    int nb = 1;
    std::vector<std::string> domains;
    for (const auto& k : keys) {
        domains.push_back(catalogTable(k.table).col(k.column).domain);
        nb *= (int)domains.back().size();
    }
    if (nb > 64) throw std::runtime_error("analyzed plan: more than 64 groups for a keyed aggregate");
    // bucket = mixed radix over the keys in GROUP BY order, each key's index
    // in its value set (the reference's order: metal_plan_builder.cpp:335);
    // a value outside the set lands beyond the buckets: a bounds error
    std::string bucket;
    int radix = nb;
    for (size_t j = 0; j < keys.size(); j++) {
        radix /= (int)domains[j].size();
        std::string idx = std::to_string(nb);
        for (int v = (int)domains[j].size() - 1; v >= 0; --v)
            idx = "(" + keys[j].column + "[i] == '" + std::string(1, domains[j][v]) + "' ? " + std::to_string(v) +
                  " : " + idx + ")";
        bucket += (bucket.empty() ? "" : " + ") + std::string("(") + idx + ") * " + std::to_string(radix);
    }
    std::vector<ResolvedColumn> cols(keys.begin(), keys.end());
    for (const auto& f : aq.filters) collectColumns(f, cols);
    struct Slot {
        std::string name, code;
        bool wide;
        int scale;
    };
    std::vector<Slot> slots;
    std::vector<CudaResultSchema::DerivedColumn> derived;
    int countIdx = -1;
    auto needCount = [&]() {
        if (countIdx < 0) {
            countIdx = (int)slots.size();
            slots.push_back({"_count", "1", false, 0});
        }
        return slots[countIdx].name;
    };
    std::vector<std::string> outCols;
    for (size_t i = 0; i < aq.targets.size(); i++) {
        const auto& t = aq.targets[i];
        if (!t.isAgg || !t.agg) {
            auto c = plainColumn(t.expr);
            bool isKey = false;
            for (const auto& k : keys) isKey |= c && c->column == k.column && c->table == k.table;
            if (!isKey) throw std::runtime_error("analyzed plan: a non-aggregate target that is not a GROUP BY column");
            continue;
        }
        const auto& a = *t.agg;
        const std::string alias = aliasOf(t, i);
        if (a.func == AggFunc::SUM || a.func == AggFunc::AVG) {
            collectColumns(a.innerExpr, cols);
            const Lowered v = exprToCuda(a.innerExpr, "i");
            slots.push_back({a.func == AggFunc::SUM ? alias : "_sum_" + alias, v.code, true, v.scale});
            if (a.func == AggFunc::AVG) derived.push_back({alias, slots.back().name, needCount()});
        } else if (a.func == AggFunc::COUNT) {
            if (countIdx >= 0 && slots[countIdx].name == "_count") slots[countIdx].name = alias;
            else if (countIdx < 0) {
                countIdx = (int)slots.size();
                slots.push_back({alias, "1", false, 0});
            } else {
                slots.push_back({alias, "1", false, 0});
            }
        } else {
            throw std::runtime_error("analyzed plan: " + aggName(a.func) + " in a keyed aggregate");
        }
    }
    // derived columns named the count slot before a COUNT target may have renamed it
    for (auto& d : derived)
        if (d.denominator == "_count" && countIdx >= 0) d.denominator = slots[countIdx].name;
    int vpb = 0;
    std::vector<int> offs;
    for (const auto& sl : slots) {
        offs.push_back(vpb);
        vpb += sl.wide ? 2 : 1;
    }
    auto scan = scanFor(plan, table, cols, tune);
    auto f = selectIf(std::move(scan), combineFilters(aq.filters, "i"));
    auto agg = std::make_unique<CudaKeyedAgg>(std::move(f), "d_ir_keyed", bucket, nb, vpb);
    for (size_t j = 0; j < slots.size(); j++) agg->addAggregate(slots[j].name, offs[j], slots[j].code, "add", slots[j].wide, slots[j].scale);
    if (tune.keyedStrategy) agg->setStrategy((CudaKeyedAgg::Strategy)tune.keyedStrategy);
    appendPhase(plan, plan.name + "_reduce", std::move(agg), tune);
    plan.chunkable = true;
    plan.decorate.push_back([keyNames, domains, nb, derived](CudaResultSchema& rs) {
        int radix = nb;
        rs.keyedAgg.keys.clear();
        for (size_t j = 0; j < keyNames.size(); j++) {
            radix /= (int)domains[j].size();
            std::vector<std::string> labels;
            for (char ch : domains[j]) labels.push_back(std::string(1, ch));
            rs.keyedAgg.keys.push_back({keyNames[j], radix, (int)domains[j].size(), labels});
        }
        rs.keyedAgg.derived = derived;
    });
    return plan;
}

// One table, GROUP BY one integer column (the Q18 shape).
CudaQueryPlan planHashGroupBy(const AnalyzedQuery& aq, const std::string& table, const ResolvedColumn& key,
                              const std::string& keyName, const std::string& name, const TuneConfig& tune) {
    CudaQueryPlan plan;
    plan.name = name.empty() ? "HASH_GROUPBY" : name;
    std::vector<ResolvedColumn> cols{key};
    for (const auto& f : aq.filters) collectColumns(f, cols);
    std::vector<std::pair<std::string, std::string>> aggs;
    for (size_t i = 0; i < aq.targets.size(); i++) {
        const auto& t = aq.targets[i];
        if (!t.isAgg || !t.agg) {
            auto c = plainColumn(t.expr);
            if (!c || c->column != key.column) throw std::runtime_error("analyzed plan: a non-aggregate target that is not the GROUP BY column");
            continue;
        }
        const auto& a = *t.agg;
        if (a.func == AggFunc::SUM) {
            collectColumns(a.innerExpr, cols);
            aggs.emplace_back(aliasOf(t, i), exprToCuda(a.innerExpr, "i").code);
        } else if (a.func == AggFunc::COUNT) {
            aggs.emplace_back(aliasOf(t, i), "1");
        } else {
            throw std::runtime_error("analyzed plan: " + aggName(a.func) + " in a hash group-by");
        }
    }
    auto scan = scanFor(plan, table, cols, tune);
    auto f = selectIf(std::move(scan), combineFilters(aq.filters, "i"));
    // every row may be its own group: the table is sized by the row count
    auto gb = std::make_unique<CudaHashGroupBy>(std::move(f), "irg", "(long long)" + key.column + "[i]", "long long",
                                                "2 * max(n_" + table + ", 1)", tune.hashLayout, tune.maxProbe);
    for (const auto& [n, v] : aggs) gb->addAggregate(n, v);
    gb->setWarpAggregate(tune.warpAggregate);
    gb->setSharedPreAgg(tune.smemPreAggLog2, tune.smemProbe);
    appendPhase(plan, plan.name + "_aggregate", std::move(gb), tune);
    plan.decorate.push_back([keyName](CudaResultSchema& rs) { rs.hashAgg.keyName = keyName; });
    return plan;
}

// dim JOIN probe ON b_key = p_fk (the Q3 shape).
CudaQueryPlan planJoin(const AnalyzedQuery& aq, const TuneConfig& tune) {
    if (aq.joins.size() != 1) throw std::runtime_error("analyzed plan: joins of two tables on one key are planned");
    const auto& j = aq.joins[0];
    const ResolvedColumn l = resolveColumn(j.leftTable, j.leftCol), r = resolveColumn(j.rightTable, j.rightCol);
    const bool ok = (l.table == "dim" && l.column == "b_key" && r.table == "probe" && r.column == "p_fk") ||
                    (r.table == "dim" && r.column == "b_key" && l.table == "probe" && l.column == "p_fk");
    if (!ok) throw std::runtime_error("analyzed plan: the join is planned on dim.b_key = probe.p_fk");
    JoinAggParts jp;
    std::vector<PredPtr> bf, pf;
    for (const auto& f : aq.filters) {
        const std::string t = predicateTable(f);
        if (t == "dim") bf.push_back(f);
        else if (t == "probe") pf.push_back(f);
        else throw std::runtime_error("analyzed plan: a filter on neither joined table");
    }
    jp.buildPred = combineFilters(bf, "i");
    jp.probePred = combineFilters(pf, "i");
    if (aq.groupBy.size() != 1) throw std::runtime_error("analyzed plan: the join groups by its key");
    auto g = plainColumn(aq.groupBy[0]);
    if (!g || !((g->table == "probe" && g->column == "p_fk") || (g->table == "dim" && g->column == "b_key")))
        throw std::runtime_error("analyzed plan: the join groups by its key (p_fk / b_key)");
    std::string sumAlias;
    int nsum = 0;
    for (size_t i = 0; i < aq.targets.size(); i++) {
        const auto& t = aq.targets[i];
        if (!t.isAgg || !t.agg) continue;
        if (t.agg->func != AggFunc::SUM) throw std::runtime_error("analyzed plan: the join aggregates one SUM");
        std::vector<ResolvedColumn> cols;
        collectColumns(t.agg->innerExpr, cols);
        for (const auto& c : cols)
            if (c.table != "probe" || (c.column != "p_price" && c.column != "p_discount"))
                throw std::runtime_error("analyzed plan: the join's SUM reads probe price / discount");
        jp.revenue = exprToCuda(t.agg->innerExpr, "i").code;
        sumAlias = aliasOf(t, i);
        nsum++;
    }
    if (nsum != 1) throw std::runtime_error("analyzed plan: the join aggregates one SUM");
    jp.k = 0;
    if (aq.limit >= 0) {
        if (aq.limit < 1 || aq.limit > 32) throw std::runtime_error("analyzed plan: LIMIT must be in [1, 32] for the GPU top-k");
        if (aq.orderBy.empty() || !aq.orderBy[0].descending ||
            !(isAliasRef(aq.orderBy[0].expr, sumAlias) || aq.orderBy.size() > 2))
            throw std::runtime_error("analyzed plan: LIMIT needs ORDER BY the SUM DESC (ties by key ASC)");
        if (aq.orderBy.size() == 2) {
            auto k2 = plainColumn(aq.orderBy[1].expr);
            if (!k2 || aq.orderBy[1].descending || !(k2->column == "p_fk" || k2->column == "b_key"))
                throw std::runtime_error("analyzed plan: ties are broken by the key ascending");
        }
        jp.k = aq.limit;
    }
    CudaQueryPlan plan = buildJoinAgg(jp, tune);
    plan.decorate.push_back([sumAlias](CudaResultSchema& rs) {
        rs.topk.valueName = sumAlias;
        if (!rs.hashAgg.aggs.empty()) rs.hashAgg.aggs[0].name = sumAlias;
    });
    if (plan.cpuSort) plan.cpuSort->keys[0].column = sumAlias;
    return plan;
}

}  // namespace

CudaQueryPlan buildCudaPlan(const ir::AnalyzedQuery& aq, const std::string& queryName, const TuneConfig& tune) {
    if (aq.tables.empty()) throw std::runtime_error("analyzed plan: no table");
    for (char ch : queryName)
        if (!(std::isalnum((unsigned char)ch) || ch == '_'))
            throw std::runtime_error("analyzed plan: the query name becomes a kernel name: letters, digits, '_'");
    if (!aq.hasAggregation()) throw std::runtime_error("analyzed plan: only aggregating queries are planned");
    CudaQueryPlan plan;
    if (aq.tables.size() == 2 || !aq.joins.empty()) {
        plan = planJoin(aq, tune);
    } else if (aq.isSingleTable()) {
        const std::string table = resolveTable(aq.tables[0]);
        catalogTable(table);  // throws on an unknown table
        if (!aq.hasGroupBy()) {
            if (!aq.orderBy.empty() || aq.limit >= 0)
                throw std::runtime_error("analyzed plan: ORDER BY / LIMIT of a one-row aggregate");
            plan = planScalarAgg(aq, table, queryName, tune);
        } else {
            std::vector<ResolvedColumn> keys;
            std::vector<std::string> names;
            bool allDomains = true;
            for (const auto& g : aq.groupBy) {
                auto c = plainColumn(g);
                if (!c || c->table != table) throw std::runtime_error("analyzed plan: GROUP BY a column of the table");
                keys.push_back(*c);
                names.push_back(std::get<ColRef>(g->node).column);
                allDomains &= !catalogTable(c->table).col(c->column).domain.empty();
            }
            if (!aq.orderBy.empty() || aq.limit >= 0)
                throw std::runtime_error("analyzed plan: ORDER BY / LIMIT of a group-by is planned for joins only");
            if (allDomains) plan = planKeyedAgg(aq, table, keys, names, queryName, tune);
            else if (keys.size() == 1 && keys[0].cudaType != "unsigned char")
                plan = planHashGroupBy(aq, table, keys[0], names[0], queryName, tune);
            else throw std::runtime_error("analyzed plan: GROUP BY several columns needs known value sets");
        }
    } else {
        throw std::runtime_error("analyzed plan: more than two tables");
    }
    if (!queryName.empty()) plan.name = queryName;
    plan.spec = "analyzed=" + (queryName.empty() ? plan.name : queryName);
    return plan;
}

CudaCodegen generateFromPlan(const CudaQueryPlan& plan) {
    CudaCodegen cg;
    for (const auto& h : plan.helpers) cg.addHelper(h);
    for (const auto& ph : plan.phases) {
        cg.beginPhase(ph.name);
        cg.setPhaseThreadgroupSize(ph.threadgroupSize);
        cg.setPhaseSingleThread(ph.singleThread);
        cg.setPhaseMinBlocksPerSM(ph.minBlocksPerSM);
        cg.setPhaseSmemCarveout(ph.smemCarveout);
        for (const auto& [n, sz] : ph.bitmapReads) cg.addBitmapReadParam(n, sz);
        for (const auto& [n, t] : ph.scalarParams) cg.addScalarParam(n, t);
        for (const auto& ss : ph.sizeScalars) cg.addSizeScalarParam(ss.name, ss.type, ss.expr);
        for (const auto& eb : ph.extraBuffers) {
            if (eb.readOnly) cg.addReadBufferParam(eb.name, eb.type);
            else cg.addBufferParam(eb.name, eb.type, "", eb.zeroInit);
        }
        for (const auto& line : ph.prologue) cg.addLine(line);
        if (ph.root) ph.root->produce(cg, []() {});
        cg.endPhase();
    }
    for (const auto& d : plan.decorate) d(cg.resultSchema());
    return cg;
}

long long planAlgorithmicBytes(const CudaQueryPlan& plan, const std::map<std::string, long long>& rows) {
    CudaCodegen cg = generateFromPlan(plan);
    long long bytes = 0;
    for (const auto& ph : cg.getPhases()) {
        std::set<std::string> seen;
        for (const auto& b : ph.bindings) {
            if (b.kind != CudaParamKind::TableData || !seen.insert(b.name).second) continue;
            auto it = rows.find(b.tableName);
            if (it != rows.end()) bytes += it->second * (long long)b.elemSizeBytes();
        }
    }
    return bytes;
}

}  // namespace gpudb
