#include "param_binding.h"

#include <cctype>

namespace gpudb {

const char* paramKindName(CudaParamKind k) {
    switch (k) {
        case CudaParamKind::TableData: return "TableData";
        case CudaParamKind::TableSize: return "TableSize";
        case CudaParamKind::DeviceBuffer: return "DeviceBuffer";
        case CudaParamKind::ConstantScalar: return "ConstantScalar";
        case CudaParamKind::ConstantData: return "ConstantData";
        case CudaParamKind::ErrorWord: return "ErrorWord";
        case CudaParamKind::BufferLength: return "BufferLength";
    }
    return "?";
}

size_t cudaTypeBytes(const std::string& t) {
    if (t == "long long" || t == "unsigned long long" || t == "double" || t == "int64_t" ||
        t == "uint64_t")
        return 8;
    if (t == "unsigned char" || t == "signed char" || t == "char" || t == "bool") return 1;
    if (t == "short" || t == "unsigned short") return 2;
    if (t == "int" || t == "unsigned" || t == "unsigned int" || t == "float") return 4;
    throw std::runtime_error("cudaTypeBytes: unknown element type '" + t + "'");
}

uint64_t CudaSizeResolver::getSymbol(const std::string& name) const {
    auto it = symbols_.find(name);
    if (it == symbols_.end())
        throw std::runtime_error("CudaSizeResolver: unknown symbol '" + name + "'");
    return it->second;
}

namespace {

// Recursive-descent evaluator over unsigned 64-bit arithmetic.
struct Parser {
    const std::string& s;
    const CudaSizeResolver& r;
    size_t p = 0;

    void ws() {
        while (p < s.size() && std::isspace((unsigned char)s[p])) p++;
    }
    [[noreturn]] void fail(const std::string& why) {
        throw std::runtime_error("CudaSizeResolver: cannot resolve '" + s + "': " + why);
    }
    bool eat(char c) {
        ws();
        if (p < s.size() && s[p] == c) {
            p++;
            return true;
        }
        return false;
    }
    uint64_t expr() {
        uint64_t v = term();
        for (;;) {
            if (eat('+')) v += term();
            else if (eat('-')) {
                uint64_t t = term();
                v = (t > v) ? 0 : v - t;  // sizes never go negative
            } else return v;
        }
    }
    uint64_t term() {
        uint64_t v = factor();
        for (;;) {
            if (eat('*')) v *= factor();
            else if (eat('/')) {
                uint64_t d = factor();
                v = d ? v / d : 0;
            } else if (eat('%')) {
                uint64_t d = factor();
                v = d ? v % d : 0;
            } else return v;
        }
    }
    uint64_t factor() {
        ws();
        if (p >= s.size()) fail("unexpected end");
        if (eat('(')) {
            uint64_t v = expr();
            if (!eat(')')) fail("missing ')'");
            return v;
        }
        if (std::isdigit((unsigned char)s[p])) {
            uint64_t v = 0;
            while (p < s.size() && std::isdigit((unsigned char)s[p])) v = v * 10 + (s[p++] - '0');
            return v;
        }
        if (std::isalpha((unsigned char)s[p]) || s[p] == '_') {
            size_t b = p;
            while (p < s.size() && (std::isalnum((unsigned char)s[p]) || s[p] == '_')) p++;
            std::string id = s.substr(b, p - b);
            if (eat('(')) {
                std::vector<uint64_t> args{expr()};
                while (eat(',')) args.push_back(expr());
                if (!eat(')')) fail("missing ')' after call");
                return call(id, args);
            }
            if (!r.hasSymbol(id)) fail("unknown symbol '" + id + "'");
            return r.getSymbol(id);
        }
        fail(std::string("unexpected '") + s[p] + "'");
    }
    uint64_t call(const std::string& f, const std::vector<uint64_t>& a) {
        if (f == "pow2ceil" && a.size() == 1) {
            uint64_t v = 1;
            while (v < a[0]) v <<= 1;
            return v;
        }
        if (f == "log2ceil" && a.size() == 1) {
            uint64_t l = 0;
            while ((uint64_t(1) << l) < a[0]) l++;
            return l;
        }
        if (f == "max" && a.size() == 2) return a[0] > a[1] ? a[0] : a[1];
        if (f == "min" && a.size() == 2) return a[0] < a[1] ? a[0] : a[1];
        fail("unknown function '" + f + "'");
    }
};

}  // namespace

uint64_t CudaSizeResolver::resolve(const std::string& expr) const {
    Parser ps{expr, *this};
    ps.ws();
    if (ps.p >= expr.size()) throw std::runtime_error("CudaSizeResolver: empty expression");
    uint64_t v = ps.expr();
    ps.ws();
    if (ps.p != expr.size()) ps.fail("trailing characters");
    return v;
}

}  // namespace gpudb
