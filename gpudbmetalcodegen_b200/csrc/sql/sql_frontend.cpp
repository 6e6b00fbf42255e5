#include "sql_frontend.h"

#include <algorithm>
#include <cctype>
#include <map>
#include <memory>
#include <set>
#include <stdexcept>
#include <vector>

namespace gpudb {

namespace {

// ---- tokens -----------------------------------------------------------
struct Tok {
    enum Kind { Ident, Number, String, Symbol, End } kind;
    std::string text;  // identifiers lower-cased
    long long num = 0;
};

std::vector<Tok> tokenize(const std::string& s) {
    std::vector<Tok> out;
    size_t i = 0;
    while (i < s.size()) {
        const char c = s[i];
        if (std::isspace((unsigned char)c)) {
            ++i;
        } else if (c == '-' && i + 1 < s.size() && s[i + 1] == '-') {
            while (i < s.size() && s[i] != '\n') ++i;  // comment
        } else if (std::isalpha((unsigned char)c) || c == '_') {
            size_t j = i;
            while (j < s.size() && (std::isalnum((unsigned char)s[j]) || s[j] == '_')) ++j;
            std::string t = s.substr(i, j - i);
            for (auto& ch : t) ch = (char)std::tolower((unsigned char)ch);
            out.push_back({Tok::Ident, t});
            i = j;
        } else if (std::isdigit((unsigned char)c)) {
            size_t j = i;
            while (j < s.size() && std::isdigit((unsigned char)s[j])) ++j;
            if (j < s.size() && s[j] == '.')
                throw std::runtime_error("sql: decimal literal at '" + s.substr(i, j - i + 2) +
                                         "': write constants in the column's integer units");
            Tok t{Tok::Number, s.substr(i, j - i)};
            t.num = std::stoll(t.text);
            out.push_back(t);
            i = j;
        } else if (c == '\'') {
            const size_t j = s.find('\'', i + 1);
            if (j == std::string::npos) throw std::runtime_error("sql: unterminated string");
            out.push_back({Tok::String, s.substr(i + 1, j - i - 1)});
            i = j + 1;
        } else {
            static const char* two[] = {"<=", ">=", "<>", "!="};
            std::string sym(1, c);
            for (const char* t : two)
                if (s.compare(i, 2, t) == 0) sym = t;
            if (sym.size() == 1 && std::string("=<>*+-/%(),;").find(c) == std::string::npos)
                throw std::runtime_error(std::string("sql: unexpected character '") + c + "'");
            if (sym == "!=") sym = "<>";
            out.push_back({Tok::Symbol, sym});
            i += (sym == "<>" && s[i] == '!') ? 2 : sym.size();
        }
    }
    out.push_back({Tok::End, ""});
    return out;
}

// ---- expressions --------------------------------------------------------
struct Expr {
    enum Kind { Col, Num, Str, Bin, Func } kind = Col;
    std::string name;  // column / function name, operator
    long long num = 0;
    bool star = false;  // count(*)
    std::vector<std::shared_ptr<Expr>> args;
    // Canonical text: fully parenthesised, no spaces.
    std::string canon() const {
        switch (kind) {
            case Col: return name;
            case Num: return std::to_string(num);
            case Str: return "'" + name + "'";
            case Bin: return "(" + args[0]->canon() + name + args[1]->canon() + ")";
            case Func: {
                if (star) return name + "(*)";
                std::string s = name + "(";
                for (size_t i = 0; i < args.size(); i++) s += (i ? "," : "") + args[i]->canon();
                return s + ")";
            }
        }
        return "";
    }
};
using P = std::shared_ptr<Expr>;

P node(Expr::Kind k, const std::string& name) {
    auto e = std::make_shared<Expr>();
    e->kind = k;
    e->name = name;
    return e;
}

struct Pred {
    P lhs, rhs;
    std::string op;
};

struct Select {
    std::vector<std::pair<P, std::string>> items;  // expression, alias
    std::vector<std::string> from;
    std::vector<Pred> where;
    std::vector<P> groupBy;
    std::vector<std::pair<P, bool>> orderBy;  // expression, descending
    long long limit = -1;
};

class Parser {
public:
    explicit Parser(std::vector<Tok> t) : t_(std::move(t)) {}

    Select parse() {
        Select q;
        expectWord("select");
        do {
            P e = expr();
            std::string alias;
            if (isWord("as")) {
                ++p_;
                alias = ident();
            } else if (t_[p_].kind == Tok::Ident && !keyword(t_[p_].text)) {
                alias = ident();
            }
            q.items.push_back({e, alias});
        } while (sym(","));
        expectWord("from");
        do q.from.push_back(ident());
        while (sym(","));
        if (isWord("where")) {
            ++p_;
            do q.where.push_back(pred());
            while (word("and"));
            if (isWord("or")) throw std::runtime_error("sql: OR is not supported; predicates are a conjunction");
        }
        if (isWord("group")) {
            ++p_;
            expectWord("by");
            do q.groupBy.push_back(expr());
            while (sym(","));
        }
        if (isWord("order")) {
            ++p_;
            expectWord("by");
            do {
                P e = expr();
                bool desc = false;
                if (word("desc")) desc = true;
                else word("asc");
                q.orderBy.push_back({e, desc});
            } while (sym(","));
        }
        if (word("limit")) {
            if (t_[p_].kind != Tok::Number) throw std::runtime_error("sql: LIMIT needs an integer");
            q.limit = t_[p_++].num;
        }
        sym(";");
        if (t_[p_].kind != Tok::End) throw std::runtime_error("sql: unexpected '" + t_[p_].text + "'");
        return q;
    }

private:
    static bool keyword(const std::string& w) {
        static const std::set<std::string> k = {"from", "where", "group", "order", "by", "limit", "and", "or",
                                                "as", "asc", "desc", "between", "select"};
        return k.count(w) > 0;
    }
    bool isWord(const char* w) const { return t_[p_].kind == Tok::Ident && t_[p_].text == w; }
    bool word(const char* w) {
        if (!isWord(w)) return false;
        ++p_;
        return true;
    }
    void expectWord(const char* w) {
        if (!word(w)) throw std::runtime_error(std::string("sql: expected ") + w + " at '" + t_[p_].text + "'");
    }
    bool sym(const char* s) {
        if (t_[p_].kind == Tok::Symbol && t_[p_].text == s) {
            ++p_;
            return true;
        }
        return false;
    }
    std::string ident() {
        if (t_[p_].kind != Tok::Ident || keyword(t_[p_].text))
            throw std::runtime_error("sql: expected a name at '" + t_[p_].text + "'");
        return t_[p_++].text;
    }
    Pred pred() {
        P l = expr();
        if (word("between")) {
            P lo = expr();
            expectWord("and");
            P hi = expr();
            // a BETWEEN lo AND hi: two predicates; the second is queued
            pending_.push_back({l, hi, "<="});
            return {l, lo, ">="};
        }
        static const char* ops[] = {"<=", ">=", "<>", "=", "<", ">"};
        for (const char* o : ops)
            if (sym(o)) return {l, expr(), o};
        throw std::runtime_error("sql: expected a comparison at '" + t_[p_].text + "'");
    }
    P expr() {
        P l = term();
        while (t_[p_].kind == Tok::Symbol && (t_[p_].text == "+" || t_[p_].text == "-")) {
            const std::string op = t_[p_++].text;
            l = bin(op, l, term());
        }
        return l;
    }
    P term() {
        P l = factor();
        while (t_[p_].kind == Tok::Symbol && (t_[p_].text == "*" || t_[p_].text == "/" || t_[p_].text == "%")) {
            const std::string op = t_[p_++].text;
            l = bin(op, l, factor());
        }
        return l;
    }
    P factor() {
        const Tok& t = t_[p_];
        if (t.kind == Tok::Number) {
            ++p_;
            auto e = node(Expr::Num, "");
            e->num = t.num;
            return e;
        }
        if (t.kind == Tok::String) {
            ++p_;
            return node(Expr::Str, t.text);
        }
        if (sym("-")) {
            P f = factor();
            if (f->kind != Expr::Num) throw std::runtime_error("sql: unary minus applies to constants only");
            f->num = -f->num;
            return f;
        }
        if (sym("(")) {
            P e = expr();
            if (!sym(")")) throw std::runtime_error("sql: expected ')'");
            return e;
        }
        const std::string name = ident();
        if (sym("(")) {
            auto e = node(Expr::Func, name);
            if (sym("*")) {
                e->star = true;
            } else {
                do e->args.push_back(expr());
                while (sym(","));
            }
            if (!sym(")")) throw std::runtime_error("sql: expected ')' after the arguments of " + name);
            return e;
        }
        return node(Expr::Col, name);
    }
    static P bin(const std::string& op, P l, P r) {
        auto e = node(Expr::Bin, op);
        e->args = {std::move(l), std::move(r)};
        return e;
    }

    std::vector<Tok> t_;
    size_t p_ = 0;

public:
    std::vector<Pred> pending_;  // second halves of BETWEEN
};

// ---- analysis -----------------------------------------------------------
// A predicate "column op constant" (constant on either side).
struct Bound {
    std::string col, op;
    long long value;
};

std::string flip(const std::string& op) {
    if (op == "<") return ">";
    if (op == ">") return "<";
    if (op == "<=") return ">=";
    if (op == ">=") return "<=";
    return op;
}

class Analysis {
public:
    explicit Analysis(Select q) : q_(std::move(q)) {
        for (const auto& p : q_.where) {
            const bool lc = p.lhs->kind == Expr::Col, rc = p.rhs->kind == Expr::Col;
            if (lc && rc) {
                if (p.op != "=") throw std::runtime_error("sql: a column-to-column predicate must be an equality");
                joins_.push_back({p.lhs->name, p.rhs->name});
            } else if (lc && p.rhs->kind == Expr::Num) {
                bounds_.push_back({p.lhs->name, p.op, p.rhs->num});
            } else if (rc && p.lhs->kind == Expr::Num) {
                bounds_.push_back({p.rhs->name, flip(p.op), p.lhs->num});
            } else {
                throw std::runtime_error("sql: unsupported predicate on " + p.lhs->canon());
            }
        }
    }

    std::string spec() {
        std::set<std::string> from(q_.from.begin(), q_.from.end());
        if (from == std::set<std::string>{"fact"}) return fact();
        if (from == std::set<std::string>{"dim", "probe"}) return semiJoin();
        if (from == std::set<std::string>{"zprobe"}) return groupBy();
        if (from == std::set<std::string>{"zbuild", "zprobe"}) return hashJoin();
        if (from == std::set<std::string>{"mix"}) return mix();
        if (from == std::set<std::string>{"mix", "mixdim"}) return mixJoin();
        throw std::runtime_error("sql: no plan template reads the tables of this query");
    }

private:
    // The constant of the predicate `col op value`, consumed once; for
    // integer columns, `> v` is `>= v + 1` and `<= v` is `< v + 1`.
    bool take(const std::string& col, const std::string& op, long long& v) {
        for (size_t i = 0; i < bounds_.size(); i++) {
            auto& b = bounds_[i];
            if (b.col != col) continue;
            long long x;
            if (b.op == op) x = b.value;
            else if (op == "<" && b.op == "<=") x = b.value + 1;
            else if (op == "<=" && b.op == "<") x = b.value - 1;
            else if (op == ">" && b.op == ">=") x = b.value - 1;
            else if (op == ">=" && b.op == ">") x = b.value + 1;
            else continue;
            v = x;
            bounds_.erase(bounds_.begin() + (long)i);
            return true;
        }
        return false;
    }
    long long need(const std::string& col, const std::string& op, const char* what) {
        long long v;
        if (!take(col, op, v))
            throw std::runtime_error(std::string("sql: the ") + what + " needs a predicate " + col + " " + op + " <constant>");
        return v;
    }
    void noneLeft(const char* what) const {
        if (!bounds_.empty())
            throw std::runtime_error(std::string("sql: the ") + what + " has no predicate like " + bounds_[0].col + " " +
                                     bounds_[0].op + " " + std::to_string(bounds_[0].value));
    }
    std::set<std::string> groupCols() const {
        std::set<std::string> g;
        for (const auto& e : q_.groupBy) {
            if (e->kind != Expr::Col) throw std::runtime_error("sql: GROUP BY takes columns");
            g.insert(e->name);
        }
        return g;
    }
    void itemsIn(const std::set<std::string>& allowed, const char* what) const {
        for (const auto& it : q_.items)
            if (!allowed.count(it.first->canon()))
                throw std::runtime_error(std::string("sql: the ") + what + " does not compute " + it.first->canon());
    }
    // The template returns its rows ordered by these columns ascending, so
    // ORDER BY may only ask for that (or a prefix of it), and no LIMIT.
    void orderedBy(const std::vector<std::string>& cols, const char* what) const {
        if (q_.limit >= 0) throw std::runtime_error(std::string("sql: the ") + what + " takes no LIMIT");
        for (size_t i = 0; i < q_.orderBy.size(); i++) {
            const auto& o = q_.orderBy[i];
            if (i >= cols.size() || o.first->kind != Expr::Col || o.second ||
                std::find(cols.begin(), cols.end(), o.first->name) == cols.end())
                throw std::runtime_error(std::string("sql: the ") + what + " is ordered by its key columns ascending");
        }
    }
    bool joined(const std::string& a, const std::string& b) const {
        for (const auto& j : joins_)
            if ((j.first == a && j.second == b) || (j.first == b && j.second == a)) return true;
        return false;
    }

    std::string fact() {
        if (!joins_.empty()) throw std::runtime_error("sql: fact takes no join predicate");
        if (groupCols() == std::set<std::string>{"f_flag_a", "f_flag_b"}) {
            itemsIn({"f_flag_a", "f_flag_b", "sum(f_quantity)", "sum(f_price)", "sum((f_price*(100-f_discount)))",
                     "sum(((f_price*(100-f_discount))*(100+f_tax)))", "sum(f_discount)", "avg(f_quantity)",
                     "avg(f_price)", "avg(f_discount)", "count(*)"},
                    "Q1-shape aggregate");
            const long long le = need("f_ship_day", "<=", "Q1-shape aggregate");
            noneLeft("Q1-shape aggregate");
            orderedBy({"f_flag_a", "f_flag_b"}, "Q1-shape aggregate");
            return "template=q1;ship_le=" + std::to_string(le);
        }
        if (q_.groupBy.empty()) {
            itemsIn({"sum((f_price*f_discount))"}, "Q6-shape sum");
            const long long ge = need("f_ship_day", ">=", "Q6-shape sum");
            const long long lt = need("f_ship_day", "<", "Q6-shape sum");
            const long long lo = need("f_discount", ">=", "Q6-shape sum");
            const long long hi = need("f_discount", "<=", "Q6-shape sum");
            const long long q = need("f_quantity", "<", "Q6-shape sum");
            noneLeft("Q6-shape sum");
            orderedBy({}, "Q6-shape sum");
            return "template=q6;ship_ge=" + std::to_string(ge) + ";ship_lt=" + std::to_string(lt) +
                   ";disc_lo=" + std::to_string(lo) + ";disc_hi=" + std::to_string(hi) + ";qty_lt=" + std::to_string(q);
        }
        throw std::runtime_error("sql: fact is grouped by (f_flag_a, f_flag_b) or not at all");
    }

    std::string semiJoin() {
        if (!joined("b_key", "p_fk") || joins_.size() != 1)
            throw std::runtime_error("sql: dim and probe join on b_key = p_fk");
        const std::string w = "dim/probe join";
        const long long seg = need("b_segment", "=", w.c_str());
        const long long od = need("b_order_day", "<", w.c_str());
        const long long ship = need("p_ship_day", ">", w.c_str());
        noneLeft(w.c_str());
        const std::string consts =
            ";seg=" + std::to_string(seg) + ";od_lt=" + std::to_string(od) + ";ship_gt=" + std::to_string(ship);
        const std::string rev = "sum((p_price*(100-p_discount)))";
        if (groupCols() == std::set<std::string>{"p_fk"}) {
            itemsIn({"p_fk", "b_key", rev}, "grouped join");
            // ORDER BY the revenue (or its alias) descending, then the key ascending
            std::string alias;
            for (const auto& it : q_.items)
                if (it.first->canon() == rev) alias = it.second;
            if (q_.orderBy.empty() || !q_.orderBy[0].second ||
                !(q_.orderBy[0].first->canon() == rev ||
                  (!alias.empty() && q_.orderBy[0].first->kind == Expr::Col && q_.orderBy[0].first->name == alias)))
                throw std::runtime_error("sql: the grouped join orders by its revenue descending");
            for (size_t i = 1; i < q_.orderBy.size(); i++) {
                const std::string c = q_.orderBy[i].first->canon();
                if ((c != "p_fk" && c != "b_key") || q_.orderBy[i].second)
                    throw std::runtime_error("sql: ties of the grouped join are broken by the key ascending");
            }
            if (q_.limit < 1 || q_.limit > 32) throw std::runtime_error("sql: the grouped join needs LIMIT 1..32");
            return "template=join_topk" + consts + ";k=" + std::to_string(q_.limit);
        }
        if (q_.groupBy.empty()) {
            itemsIn({"p_fk", "b_key", "(p_price*(100-p_discount))"}, "join output");
            if (!q_.orderBy.empty() || q_.limit >= 0)
                throw std::runtime_error("sql: the join output is unordered and unlimited");
            return "template=join_rows" + consts;
        }
        throw std::runtime_error("sql: the join is grouped by p_fk or not at all");
    }

    std::string groupBy() {
        if (!joins_.empty() || !bounds_.empty()) throw std::runtime_error("sql: the zprobe group-by takes no predicate");
        if (groupCols() != std::set<std::string>{"z_key"}) throw std::runtime_error("sql: zprobe is grouped by z_key");
        itemsIn({"z_key", "count(*)", "sum(z_value)"}, "zprobe group-by");
        orderedBy({"z_key"}, "zprobe group-by");
        return "template=groupby";
    }

    std::string hashJoin() {
        if (!joined("zb_key", "z_key") || joins_.size() != 1 || !bounds_.empty())
            throw std::runtime_error("sql: zbuild and zprobe join on zb_key = z_key only");
        const auto g = groupCols();
        if (g != std::set<std::string>{"z_key"} && g != std::set<std::string>{"zb_key"})
            throw std::runtime_error("sql: the hash join is grouped by its key");
        itemsIn({"z_key", "zb_key", "count(*)", "sum(zb_payload)"}, "hash join");
        orderedBy({"z_key", "zb_key"}, "hash join");
        return "template=hashjoin";
    }

    // The mixed-workload templates over `mix` (the batch path's query
    // shapes): filtered count + sum, grouped by key % card, top-k of it.
    std::string mix() {
        if (!joins_.empty()) throw std::runtime_error("sql: mix takes no join predicate");
        const long long thr = need("m_filter", "<", "mix query");
        noneLeft("mix query");
        const std::string t = ";thr=" + std::to_string(thr);
        if (q_.groupBy.empty()) {
            itemsIn({"count(*)", "sum(m_value)"}, "filtered aggregate");
            orderedBy({}, "filtered aggregate");
            return "template=mix_agg" + t;
        }
        // GROUP BY <key column> % <card>
        const P g = q_.groupBy.size() == 1 ? q_.groupBy[0] : nullptr;
        if (!g || g->kind != Expr::Bin || g->name != "%" || g->args[0]->kind != Expr::Col ||
            g->args[1]->kind != Expr::Num || g->args[1]->num < 1 ||
            (g->args[0]->name != "m_rank_u" && g->args[0]->name != "m_rank_z"))
            throw std::runtime_error("sql: mix is grouped by m_rank_u % <card> or m_rank_z % <card>");
        const std::string key = g->args[0]->name, gk = g->canon();
        const long long card = g->args[1]->num;
        itemsIn({gk, "count(*)", "sum(m_value)"}, "mix group-by");
        const std::string base = ";key=" + key + ";card=" + std::to_string(card) + t + ";groups=" + std::to_string(card);
        if (q_.limit < 0) {
            orderedBy({}, "mix group-by");
            return "template=mix_groupby" + base;
        }
        if (q_.limit < 1 || q_.limit > 32) throw std::runtime_error("sql: the mix top-k needs LIMIT 1..32");
        if (q_.orderBy.empty() || q_.orderBy[0].first->canon() != "sum(m_value)" || !q_.orderBy[0].second)
            throw std::runtime_error("sql: the mix top-k orders by sum(m_value) descending");
        for (size_t i = 1; i < q_.orderBy.size(); i++)
            if (q_.orderBy[i].first->canon() != gk || q_.orderBy[i].second)
                throw std::runtime_error("sql: ties of the mix top-k are broken by the group key ascending");
        return "template=mix_topk" + base + ";k=" + std::to_string(q_.limit);
    }

    std::string mixJoin() {
        if (!joined("m_fk", "md_key") || joins_.size() != 1)
            throw std::runtime_error("sql: mix and mixdim join on m_fk = md_key");
        const long long thr = need("m_filter", "<", "mix join");
        const long long attr = need("md_attr", "<", "mix join");
        noneLeft("mix join");
        if (!q_.groupBy.empty()) throw std::runtime_error("sql: the mix join is not grouped");
        itemsIn({"count(*)", "sum(m_value)"}, "mix join");
        orderedBy({}, "mix join");
        return "template=mix_join;thr=" + std::to_string(thr) + ";attr_lt=" + std::to_string(attr);
    }

    Select q_;
    std::vector<std::pair<std::string, std::string>> joins_;
    std::vector<Bound> bounds_;
};

}  // namespace

std::string sqlToSpec(const std::string& sql) {
    Parser p(tokenize(sql));
    Select q = p.parse();
    for (auto& extra : p.pending_) q.where.push_back(extra);
    return Analysis(std::move(q)).spec();
}

}  // namespace gpudb
