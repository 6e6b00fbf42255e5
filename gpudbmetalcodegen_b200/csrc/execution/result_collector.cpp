#include "result_collector.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <sstream>
#include <stdexcept>

namespace gpudb {

std::string int128ToString(int128 v) {
    if (v == 0) return "0";
    const bool neg = v < 0;
    unsigned __int128 u = neg ? (unsigned __int128)(-(v + 1)) + 1 : (unsigned __int128)v;
    std::string s;
    while (u) {
        s.push_back(char('0' + (int)(u % 10)));
        u /= 10;
    }
    if (neg) s.push_back('-');
    std::reverse(s.begin(), s.end());
    return s;
}

namespace {

std::string fmt(const GenericResult::Value& v, bool exact) {
    if (auto p = std::get_if<int128>(&v)) return int128ToString(*p);
    if (auto p = std::get_if<double>(&v)) {
        char b[64];
        snprintf(b, sizeof b, exact ? "%.17g" : "%.4f", *p);
        return b;
    }
    const std::string& s = std::get<std::string>(v);
    if (s.find_first_of(",\"\n\r") == std::string::npos) return s;
    std::string q = "\"";
    for (char c : s) {
        if (c == '"') q += '"';
        q += c;
    }
    return q + "\"";
}

std::string serialise(const GenericResult& r, bool exact) {
    std::ostringstream o;
    for (size_t c = 0; c < r.columns.size(); c++) o << (c ? "," : "") << r.columns[c].name;
    o << "\n";
    for (const auto& row : r.rows) {
        for (size_t c = 0; c < row.size(); c++) o << (c ? "," : "") << fmt(row[c], exact);
        o << "\n";
    }
    return o.str();
}

// exact two-word reconstruction: total = (int64)w1 * 2^32 + w0
int128 wide(uint64_t w0, uint64_t w1) { return (int128)(int64_t)w1 * ((int128)1 << 32) + (int128)w0; }

}  // namespace

std::string GenericResult::toCanonical() const { return serialise(*this, false); }
std::string GenericResult::toExact() const { return serialise(*this, true); }

int GenericResult::columnIndex(const std::string& name) const {
    for (size_t i = 0; i < columns.size(); i++)
        if (columns[i].name == name) return (int)i;
    return -1;
}

void GenericResult::print(int limit) const {
    const std::string s = toExact();
    std::istringstream in(s);
    std::string line;
    int n = 0;
    while (std::getline(in, line)) {
        if (limit >= 0 && n > limit) {
            std::cout << "... (" << rows.size() - (size_t)limit << " more rows)\n";
            break;
        }
        std::cout << line << "\n";
        n++;
    }
}

// ------------------------------------------------------------------
// compareCanonical
// ------------------------------------------------------------------
std::string compareCanonical(const std::string& got, const std::string& expected, double absTol, double relTol) {
    auto lines = [](const std::string& s) {
        std::vector<std::string> v;
        std::istringstream in(s);
        std::string l;
        while (std::getline(in, l)) {
            if (!l.empty() && l.back() == '\r') l.pop_back();
            v.push_back(l);
        }
        while (!v.empty() && v.back().empty()) v.pop_back();
        return v;
    };
    auto csv = [](const std::string& l) {
        std::vector<std::string> out;
        std::string cur;
        bool q = false;
        for (size_t i = 0; i < l.size(); i++) {
            const char c = l[i];
            if (q) {
                if (c == '"') {
                    if (i + 1 < l.size() && l[i + 1] == '"') {
                        cur += '"';
                        i++;
                    } else q = false;
                } else cur += c;
            } else if (c == '"') q = true;
            else if (c == ',') {
                out.push_back(cur);
                cur.clear();
            } else cur += c;
        }
        out.push_back(cur);
        return out;
    };
    auto num = [](const std::string& s, double& v) {
        if (s.empty()) return false;
        char* e = nullptr;
        v = std::strtod(s.c_str(), &e);
        return e != s.c_str() && *e == '\0';
    };
    const auto a = lines(got), b = lines(expected);
    if (a.empty() && b.empty()) return "";
    if (a.empty()) return "got 0 rows, expected " + std::to_string(b.size() - 1) + " data rows";
    if (b.empty()) return "got " + std::to_string(a.size() - 1) + " data rows, expected 0";
    const auto ah = csv(a[0]), bh = csv(b[0]);
    std::vector<std::pair<size_t, size_t>> shared;
    for (size_t i = 0; i < ah.size(); i++)
        for (size_t j = 0; j < bh.size(); j++)
            if (ah[i] == bh[j]) {
                shared.push_back({i, j});
                break;
            }
    if (shared.empty()) return "schema mismatch: got cols=[" + a[0] + "] expected cols=[" + b[0] + "]";
    if (a.size() != b.size())
        return "row count mismatch: got=" + std::to_string(a.size() - 1) + " expected=" + std::to_string(b.size() - 1);
    for (size_t r = 1; r < a.size(); r++) {
        const auto ar = csv(a[r]), br = csv(b[r]);
        for (auto [i, j] : shared) {
            if (i >= ar.size() || j >= br.size() || ar[i] == br[j]) continue;
            double x, y;
            if (num(ar[i], x) && num(br[j], y)) {
                const double tol = absTol + relTol * std::max(std::fabs(x), std::fabs(y));
                if (std::fabs(x - y) <= tol) continue;
            }
            return "row " + std::to_string(r) + " col '" + ah[i] + "': " + ar[i] + " vs " + br[j];
        }
    }
    return "";
}

// ------------------------------------------------------------------
// collectors
// ------------------------------------------------------------------
GenericResult CudaResultCollector::collect(const CudaResultSchema& s, const BufferReader& read, const SizeEval& size) {
    switch (s.kind) {
        case CudaResultSchema::SCALAR_AGG: return collectScalarAgg(s, read);
        case CudaResultSchema::KEYED_AGG: return collectKeyedAgg(s, read);
        case CudaResultSchema::HASH_AGG: return collectHashAgg(s, read, size);
        case CudaResultSchema::TOPK: return collectTopK(s, read);
        case CudaResultSchema::MATERIALIZE: return collectMaterialize(s, read, size);
        case CudaResultSchema::DIRECT_AGG: return collectDirectAgg(s, read, size);
        default: return {};
    }
}

GenericResult CudaResultCollector::collectScalarAgg(const CudaResultSchema& s, const BufferReader& read) {
    GenericResult r;
    GenericResult::Row row;
    for (const auto& e : s.scalarAggs) {
        uint64_t w[2] = {0, 0};
        if (!read(e.buffer, w, e.isWide ? 16 : 8)) throw std::runtime_error("collector: missing buffer " + e.buffer);
        r.columns.push_back({e.displayName, "int"});
        row.push_back(e.isWide ? wide(w[0], w[1]) : (int128)(int64_t)w[0]);
    }
    if (!row.empty()) r.rows.push_back(std::move(row));
    return r;
}

GenericResult CudaResultCollector::collectKeyedAgg(const CudaResultSchema& s, const BufferReader& read) {
    GenericResult r;
    const auto& k = s.keyedAgg;
    std::vector<uint64_t> data((size_t)k.numBuckets * k.valuesPerBucket);
    if (!read(k.bufferName, data.data(), data.size() * 8))
        throw std::runtime_error("collector: missing buffer " + k.bufferName);
    if (k.keys.empty()) r.columns.push_back({k.bucketName, "int"});
    for (const auto& bk : k.keys) r.columns.push_back({bk.name, "string"});
    for (const auto& sl : k.slots) r.columns.push_back({sl.name, "int"});
    for (const auto& d : k.derived) r.columns.push_back({d.name, "double"});
    auto slotIndex = [&](const std::string& n) {
        for (size_t i = 0; i < k.slots.size(); i++)
            if (k.slots[i].name == n) return (int)i;
        throw std::runtime_error("collector: derived column refers to unknown slot " + n);
    };
    for (int b = 0; b < k.numBuckets; b++) {
        const uint64_t* w = data.data() + (size_t)b * k.valuesPerBucket;
        bool any = false;
        for (int v = 0; v < k.valuesPerBucket; v++) any |= (w[v] != 0);
        if (!any) continue;  // empty groups are omitted (reference collector rule)
        GenericResult::Row row;
        if (k.keys.empty()) row.push_back((int128)b);
        for (const auto& bk : k.keys) {
            const int idx = (b / bk.divisor) % bk.modulus;
            row.push_back(idx < (int)bk.labels.size() ? bk.labels[idx] : std::to_string(idx));
        }
        std::vector<int128> vals;
        for (const auto& sl : k.slots) {
            const int128 v = sl.isWide ? wide(w[sl.offset], w[sl.offset + 1]) : (int128)(int64_t)w[sl.offset];
            vals.push_back(v);
            row.push_back(v);
        }
        for (const auto& d : k.derived) {
            const int128 nu = vals[slotIndex(d.numerator)], de = vals[slotIndex(d.denominator)];
            row.push_back(de == 0 ? 0.0 : (double)nu / (double)de);
        }
        r.rows.push_back(std::move(row));
    }
    return r;
}

GenericResult CudaResultCollector::collectHashAgg(const CudaResultSchema& s, const BufferReader& read,
                                                  const SizeEval& size) {
    GenericResult r;
    const auto& h = s.hashAgg;
    const uint64_t cap = size(h.capacitySymbol);
    const bool k64 = h.keyType == "unsigned long long";
    std::vector<uint64_t> keys64;
    std::vector<uint32_t> keys32;
    std::vector<std::vector<uint64_t>> aggs(h.aggs.size(), std::vector<uint64_t>(cap));
    if (h.packedStride > 0) {
        const size_t st = (size_t)h.packedStride;
        std::vector<uint64_t> w(cap * st);
        if (!read(h.keyBuffer, w.data(), w.size() * 8)) throw std::runtime_error("collector: missing " + h.keyBuffer);
        keys64.resize(cap);
        for (uint64_t i = 0; i < cap; i++) {
            keys64[i] = ~w[i * st];  // an empty slot (0) reads as the ~0 sentinel
            for (size_t a = 0; a < h.aggs.size(); a++) aggs[a][i] = w[i * st + 1 + a];
        }
    } else if (k64) {
        keys64.resize(cap);
        if (!read(h.keyBuffer, keys64.data(), cap * 8)) throw std::runtime_error("collector: missing " + h.keyBuffer);
    } else {
        keys32.resize(cap);
        if (!read(h.keyBuffer, keys32.data(), cap * 4)) throw std::runtime_error("collector: missing " + h.keyBuffer);
    }
    for (size_t a = 0; a < h.aggs.size() && h.packedStride == 0; a++)
        if (!read(h.aggs[a].buffer, aggs[a].data(), cap * 8))
            throw std::runtime_error("collector: missing " + h.aggs[a].buffer);
    r.columns.push_back({h.keyName, "int"});
    for (const auto& a : h.aggs) r.columns.push_back({a.name, "int"});
    struct Ent {
        int64_t key;
        uint64_t slot;
    };
    std::vector<Ent> ents;
    for (uint64_t i = 0; i < cap; i++) {
        if (k64 ? keys64[i] == ~0ull : keys32[i] == 0xFFFFFFFFu) continue;
        bool any = false;
        for (const auto& a : aggs) any |= (a[i] != 0);
        if (!any) continue;  // inserted but never aggregated (e.g. unmatched build key)
        ents.push_back({k64 ? (int64_t)keys64[i] : (int64_t)(int32_t)keys32[i], i});
    }
    if (h.sortByKey) std::sort(ents.begin(), ents.end(), [](const Ent& x, const Ent& y) { return x.key < y.key; });
    r.rows.reserve(ents.size());
    for (const auto& e : ents) {
        GenericResult::Row row;
        row.push_back((int128)e.key);
        for (const auto& a : aggs) row.push_back((int128)(int64_t)a[e.slot]);
        r.rows.push_back(std::move(row));
    }
    return r;
}

GenericResult CudaResultCollector::collectTopK(const CudaResultSchema& s, const BufferReader& read) {
    GenericResult r;
    const auto& t = s.topk;
    uint64_t cnt = 0;
    if (!read(t.countBuffer, &cnt, 8)) throw std::runtime_error("collector: missing " + t.countBuffer);
    std::vector<int64_t> k(t.k), v(t.k);
    if (!read(t.keyBuffer, k.data(), 8 * (size_t)t.k) || !read(t.valueBuffer, v.data(), 8 * (size_t)t.k))
        throw std::runtime_error("collector: missing top-k output");
    r.columns = {{t.keyName, "int"}, {t.valueName, "int"}};
    std::vector<std::vector<int64_t>> extra;
    for (const auto& e : t.extra) {
        const size_t w = cudaTypeBytes(e.elementType);
        std::vector<char> raw((size_t)t.k * w);
        if (!read(e.buffer, raw.data(), raw.size())) throw std::runtime_error("collector: missing " + e.buffer);
        std::vector<int64_t> col(t.k);
        for (int i = 0; i < t.k; i++) {
            const char* p = raw.data() + (size_t)i * w;
            if (w == 8) col[i] = *(const int64_t*)p;
            else if (w == 4) col[i] = *(const int32_t*)p;
            else col[i] = *(const uint8_t*)p;
        }
        extra.push_back(std::move(col));
        r.columns.push_back({e.name, "int"});
    }
    for (uint64_t i = 0; i < cnt && i < (uint64_t)t.k; i++) {
        GenericResult::Row row{(int128)k[i], (int128)v[i]};
        for (const auto& col : extra) row.push_back((int128)col[i]);
        r.rows.push_back(std::move(row));
    }
    return r;
}

GenericResult CudaResultCollector::collectDirectAgg(const CudaResultSchema& s, const BufferReader& read,
                                                    const SizeEval& size) {
    GenericResult r;
    const auto& d = s.directAgg;
    const uint64_t n = size(d.sizeExpr);
    std::vector<std::vector<int64_t>> cols;
    r.columns.push_back({d.keyName, "int"});
    for (const auto& a : d.aggs) {
        cols.emplace_back(n);
        if (n && !read(a.buffer, cols.back().data(), n * 8)) throw std::runtime_error("collector: missing " + a.buffer);
        r.columns.push_back({a.name, "int"});
    }
    for (uint64_t i = 0; i < n; i++) {
        bool any = false;
        for (const auto& c : cols) any |= (c[i] != 0);
        if (!any) continue;  // empty bins are omitted, as for keyed aggregates
        GenericResult::Row row{(int128)i};
        for (const auto& c : cols) row.push_back((int128)c[i]);
        r.rows.push_back(std::move(row));
    }
    return r;
}

GenericResult CudaResultCollector::collectMaterialize(const CudaResultSchema& s, const BufferReader& read,
                                                      const SizeEval& size) {
    (void)size;
    GenericResult r;
    uint64_t cnt = 0;
    if (!read(s.counterBuffer, &cnt, 8)) throw std::runtime_error("collector: missing " + s.counterBuffer);
    for (const auto& c : s.columns) r.columns.push_back({c.displayName, c.elementType == "double" ? "double" : "int"});
    std::vector<std::vector<char>> cols;
    for (const auto& c : s.columns) {
        const size_t w = cudaTypeBytes(c.elementType);
        cols.emplace_back(cnt * w);
        if (cnt && !read(c.bufferName, cols.back().data(), cnt * w))
            throw std::runtime_error("collector: missing " + c.bufferName);
    }
    for (uint64_t i = 0; i < cnt; i++) {
        GenericResult::Row row;
        for (size_t c = 0; c < s.columns.size(); c++) {
            const std::string& t = s.columns[c].elementType;
            const char* p = cols[c].data() + i * cudaTypeBytes(t);
            if (t == "long long") row.push_back((int128) * (const int64_t*)p);
            else if (t == "unsigned long long") row.push_back((int128) * (const uint64_t*)p);
            else if (t == "int") row.push_back((int128) * (const int32_t*)p);
            else if (t == "unsigned" || t == "unsigned int") row.push_back((int128) * (const uint32_t*)p);
            else if (t == "unsigned char") row.push_back((int128) * (const uint8_t*)p);
            else if (t == "double") row.push_back(*(const double*)p);
            else row.push_back((int128) * (const int32_t*)p);
        }
        r.rows.push_back(std::move(row));
    }
    return r;
}

}  // namespace gpudb
