// System text -> System -> step body.
//
// Behaviour follows the reference's sysparse.cpp (parse_system_from_latex :287-393 with
// strip_env :27-68, clean_part :71-113, split_rows :115-130, lhs_var :132-173, insert_mult
// :178-251, function inlining :200-284, parse_func_defs :122-197) and the expression
// grammar / printing of codegen.cpp (:59-295), because the text a user types and the step
// body the session stores must mean the same thing in both engines. The schemes emitted
// here (Euler, Euler-Cromer, Explicit Midpoint, RK4; codegen.cpp:580-606) produce the
// reference's text byte for byte; DOPRI78 and CD bodies are accepted verbatim by the
// engine's exact form but not generated here.
#include <algorithm>
#include <cctype>
#include <cstring>
#include <regex>
#include <set>
#include <sstream>
#include <stdexcept>

#include "frontend.h"

namespace ucb {
namespace fe {

namespace {

std::string trim(const std::string& x) {
    size_t a = x.find_first_not_of(" \t\n\r");
    if (a == std::string::npos) return "";
    size_t b = x.find_last_not_of(" \t\n\r");
    return x.substr(a, b - a + 1);
}

void erase_all(std::string& s, const std::string& what) {
    size_t p;
    while ((p = s.find(what)) != std::string::npos) s.erase(p, what.size());
}

// |x| and \left| ... \right| become fabs(...).
std::string bars_to_fabs(std::string s) {
    s = std::regex_replace(s, std::regex(R"(\\left\|)"), "fabs(");
    s = std::regex_replace(s, std::regex(R"(\\right\|)"), ")");
    std::string r;
    bool opening = true;
    for (char ch : s) {
        if (ch == '|') {
            r += opening ? "fabs(" : ")";
            opening = !opening;
        } else {
            r += ch;
        }
    }
    return r;
}

// LaTeX/OCR normalisation before the equations are split.
std::string normalise(std::string s) {
    s = std::regex_replace(s, std::regex(R"(\\mathrm\s*\{([^}]*)\})"), "$1");
    s = std::regex_replace(s, std::regex(R"(\\operatorname\s*\{([^}]*)\})"), "$1");
    s = std::regex_replace(s, std::regex(R"(\\(?:bigg|Bigg|big|Big)[lr]?)"), "");
    s = std::regex_replace(s, std::regex(R"(\s*\(\s*t\s*\)\s*)"), " ");  // x(t) -> x
    s = bars_to_fabs(s);
    s = std::regex_replace(s, std::regex(R"(_\s*\{([A-Za-z0-9]+)\})"), "_$1");
    for (int pass = 0; pass < 2; ++pass) s = std::regex_replace(s, std::regex(R"((\d)\s*\.\s*(\d))"), "$1.$2");
    static const char* const kDrop[] = {"\\begin{cases}", "\\end{cases}", "\\begin{aligned}", "\\end{aligned}",
                                        "\\begin{array}", "\\end{array}", "\\left\\{", "\\right.", "\\left.", "&",
                                        "\\quad", "\\;", "\\,", "\\!", " \\ "};
    for (const char* k : kDrop) erase_all(s, k);
    s = std::regex_replace(s, std::regex(R"(\{[lcr|]+\})"), "");
    return s;
}

size_t count_char(const std::string& x, char c) { return (size_t)std::count(x.begin(), x.end(), c); }

// Removes wrapping braces, empty groups and trailing equation punctuation.
std::string strip_wrapping(std::string t) {
    t = trim(t);
    for (bool changed = true; changed;) {
        changed = false;
        size_t p;
        while ((p = t.find("{}")) != std::string::npos) {
            t.erase(p, 2);
            changed = true;
        }
        t = trim(t);
        while (!t.empty() && (t.back() == ',' || t.back() == ';' || t.back() == '.')) {
            t.pop_back();
            changed = true;
        }
        t = trim(t);
        if (t.size() >= 2 && t.front() == '{' && t.back() == '}') {
            int depth = 0;
            bool wraps = true;
            for (size_t i = 0; i < t.size(); ++i) {
                if (t[i] == '{') ++depth;
                else if (t[i] == '}') {
                    --depth;
                    if (depth == 0 && i + 1 != t.size()) {
                        wraps = false;
                        break;
                    }
                }
            }
            if (wraps) {
                t = trim(t.substr(1, t.size() - 2));
                changed = true;
            }
        }
        if (!t.empty() && t.back() == '}' && count_char(t, '}') > count_char(t, '{')) {
            t.pop_back();
            changed = true;
        }
        t = trim(t);
        if (!t.empty() && t.front() == '{' && count_char(t, '{') > count_char(t, '}')) {
            t.erase(t.begin());
            changed = true;
        }
        t = trim(t);
    }
    return t;
}

std::vector<std::string> split_on_double_backslash(const std::string& s) {
    std::vector<std::string> parts;
    size_t start = 0;
    for (size_t i = 0; i + 1 < s.size(); ++i) {
        if (s[i] == '\\' && s[i + 1] == '\\') {
            parts.push_back(s.substr(start, i - start));
            i += 1;
            start = i + 1;
        }
    }
    parts.push_back(s.substr(start));
    return parts;
}

// State variable named by an equation's left-hand side.
std::string lhs_variable(const std::string& lhs) {
    std::smatch m;
    static const std::regex dot_forms[] = {
        std::regex(R"(\\dot\s*\{\s*\\([A-Za-z]+)\s*\})"), std::regex(R"(\\dot\s*\\([A-Za-z]+))"),
        std::regex(R"(\\dot\s*\{\s*([A-Za-z]\w*)\s*\})"), std::regex(R"(\\dot\s*([A-Za-z]\w*))")};
    for (const auto& re : dot_forms) {
        if (std::regex_search(lhs, m, re)) {
            std::string base = m[1];
            const std::string tail = lhs.substr((size_t)(m.position(0) + m.length(0)));
            std::smatch mi;
            if (std::regex_search(tail, mi, std::regex(R"(_(\w+))"))) base += "_" + std::string(mi[1]);
            return base;
        }
    }
    if (std::regex_search(lhs, m, std::regex(R"(\\frac\s*\{\s*d\s*([A-Za-z]\w*)\s*\}\s*\{\s*d\s*\\?[A-Za-z]\w*\s*\})")))
        return m[1];
    if (std::regex_search(lhs, m, std::regex(R"(\\frac\s*\{\s*d\s*([A-Za-z]\w*)\s*\}\s*\{\s*d\s*\\[A-Za-z]+\s*\})")))
        return m[1];
    if (std::regex_search(lhs, m, std::regex(R"(d\s*([A-Za-z]\w*)\s*/\s*d\s*\\?[A-Za-z]\w*)"))) return m[1];
    if (std::regex_search(lhs, m, std::regex(R"(([A-Za-z]\w*)\s*')"))) return m[1];
    return "";
}

// Makes implicit products explicit ("a y" -> "a * y") using the alphabet: known names
// are matched greedily, unknown words are treated as function names.
std::string explicit_products(const std::string& rhs, const std::set<std::string>& names,
                              const std::set<std::string>& commands) {
    std::string out;
    size_t i = 0;
    bool after_operand = false;
    auto operand = [&](const std::string& tok) {
        if (after_operand) out += " * ";
        out += tok;
        after_operand = true;
    };
    while (i < rhs.size()) {
        const char c = rhs[i];
        if (std::isspace((unsigned char)c)) {
            out += c;
            ++i;
            continue;
        }
        if (c == '\\') {
            size_t j = i + 1;
            while (j < rhs.size() && std::isalpha((unsigned char)rhs[j])) ++j;
            const std::string name = rhs.substr(i + 1, j - i - 1);
            if (name == "cdot" || name == "times") {
                out += " * ";
                after_operand = false;
                i = j;
                continue;
            }
            if (commands.count(name)) {
                operand("\\" + name);
                i = j;
                continue;
            }
            if (after_operand) out += " * ";
            out += "\\" + name;
            after_operand = false;
            i = j;
            if (i < rhs.size() && rhs[i] == '^') {  // \sin^{2}: the power belongs to the function
                out += '^';
                ++i;
                if (i < rhs.size() && rhs[i] == '{') {
                    int depth = 0;
                    do {
                        out += rhs[i];
                        if (rhs[i] == '{') ++depth;
                        else if (rhs[i] == '}') --depth;
                        ++i;
                    } while (i < rhs.size() && depth > 0);
                } else if (i < rhs.size()) {
                    out += rhs[i];
                    ++i;
                }
            }
            continue;
        }
        if (std::isalpha((unsigned char)c)) {
            std::string best;
            for (size_t L = 1; i + L <= rhs.size(); ++L) {
                if (!std::isalpha((unsigned char)rhs[i + L - 1])) break;
                const std::string cand = rhs.substr(i, L);
                if (names.count(cand)) best = cand;
            }
            if (!best.empty()) {
                operand(best);
                i += best.size();
                continue;
            }
            size_t j = i;
            while (j < rhs.size() && std::isalpha((unsigned char)rhs[j])) ++j;
            const std::string word = rhs.substr(i, j - i);
            if (word == "pi") {
                operand(word);
                i = j;
                continue;
            }
            if (after_operand) out += " * ";
            out += word;
            after_operand = false;
            i = j;
            continue;
        }
        if (std::isdigit((unsigned char)c) || c == '.') {
            size_t j = i;
            while (j < rhs.size() && (std::isdigit((unsigned char)rhs[j]) || rhs[j] == '.')) ++j;
            operand(rhs.substr(i, j - i));
            i = j;
            continue;
        }
        if (c == '(') {
            if (after_operand) out += " * ";
            out += '(';
            after_operand = false;
            ++i;
            continue;
        }
        if (c == ')' || c == '}') {
            out += c;
            after_operand = true;
            ++i;
            continue;
        }
        if (c == '{') {
            out += c;
            after_operand = false;
            ++i;
            continue;
        }
        if (c == '+' || c == '-' || c == '*' || c == '/' || c == '^' || c == ',') {
            out += c;
            after_operand = false;
            ++i;
            continue;
        }
        out += c;
        ++i;
    }
    return std::regex_replace(out, std::regex("  +"), " ");
}

// One pass of auxiliary-function inlining: name(args) -> (body with (actual) args).
std::string inline_once(const std::string& expr, const FuncDefs& funcs, bool& changed) {
    std::string out;
    size_t i = 0;
    auto trimmed = [](const std::string& x) {
        size_t a = x.find_first_not_of(" \t"), b = x.find_last_not_of(" \t");
        return a == std::string::npos ? std::string() : x.substr(a, b - a + 1);
    };
    while (i < expr.size()) {
        if (std::isalpha((unsigned char)expr[i]) || expr[i] == '_') {
            size_t j = i;
            while (j < expr.size() && (std::isalnum((unsigned char)expr[j]) || expr[j] == '_')) ++j;
            const std::string name = expr.substr(i, j - i);
            size_t k = j;
            while (k < expr.size() && std::isspace((unsigned char)expr[k])) ++k;
            auto it = funcs.find(name);
            if (it != funcs.end() && k < expr.size() && expr[k] == '(') {
                int depth = 0;
                size_t p = k;
                std::vector<std::string> actual;
                std::string cur;
                for (p = k; p < expr.size(); ++p) {
                    const char c = expr[p];
                    if (c == '(') {
                        ++depth;
                        if (depth == 1) continue;
                    }
                    if (c == ')') {
                        --depth;
                        if (depth == 0) {
                            const std::string t = trimmed(cur);
                            if (!t.empty()) actual.push_back(t);
                            break;
                        }
                    }
                    if (c == ',' && depth == 1) {
                        const std::string t = trimmed(cur);
                        if (!t.empty()) actual.push_back(t);
                        cur.clear();
                        continue;
                    }
                    cur += c;
                }
                const FuncDef& def = it->second;
                if (actual.size() != def.args.size())
                    throw std::runtime_error("function " + name + ": argument count mismatch");
                std::string body = def.body;
                for (size_t ai = 0; ai < def.args.size(); ++ai) {
                    std::string rep;
                    size_t q = 0;
                    while (q < body.size()) {
                        if (std::isalpha((unsigned char)body[q]) || body[q] == '_') {
                            size_t r = q;
                            while (r < body.size() && (std::isalnum((unsigned char)body[r]) || body[r] == '_')) ++r;
                            const std::string id = body.substr(q, r - q);
                            rep += (id == def.args[ai]) ? "(" + actual[ai] + ")" : id;
                            q = r;
                        } else {
                            rep += body[q];
                            ++q;
                        }
                    }
                    body = rep;
                }
                out += "(" + body + ")";
                changed = true;
                i = p + 1;
                continue;
            }
            out += name;
            i = j;
            continue;
        }
        out += expr[i];
        ++i;
    }
    return out;
}

std::string inline_functions(const std::string& expr, const FuncDefs& funcs) {
    if (funcs.empty()) return expr;
    std::string cur = expr;
    for (int it = 0; it < 16; ++it) {
        bool changed = false;
        cur = inline_once(cur, funcs, changed);
        if (!changed) break;
    }
    return cur;
}

// ---------------------------------------------------------------- LaTeX expression grammar
const std::set<std::string>& call_names() {
    static const std::set<std::string> f = {"sin",   "cos",   "tan",  "asin", "acos", "atan", "sinh", "cosh",
                                            "tanh",  "exp",   "log",  "log2", "log10", "sqrt", "cbrt", "fabs",
                                            "abs",   "pow",   "atan2", "fmod", "floor", "ceil"};
    return f;
}
const std::map<std::string, std::string>& latex_calls() {
    static const std::map<std::string, std::string> m = {
        {"sin", "sin"},   {"cos", "cos"},   {"tan", "tan"},   {"arcsin", "asin"}, {"arccos", "acos"},
        {"arctan", "atan"}, {"sinh", "sinh"}, {"cosh", "cosh"}, {"tanh", "tanh"},   {"exp", "exp"},
        {"ln", "log"},    {"log", "log"},   {"sqrt", "sqrt"}};
    return m;
}
const std::map<std::string, std::string>& greek() {
    static const std::map<std::string, std::string> m = {
        {"alpha", "alpha"}, {"beta", "beta"},   {"gamma", "gamma"}, {"delta", "delta"},   {"epsilon", "epsilon"},
        {"varepsilon", "epsilon"}, {"zeta", "zeta"}, {"eta", "eta"}, {"theta", "theta"},  {"vartheta", "theta"},
        {"iota", "iota"},   {"kappa", "kappa"}, {"lambda", "lambda"}, {"mu", "mu"},       {"nu", "nu"},
        {"xi", "xi"},       {"pi", "pi"},       {"rho", "rho"},     {"sigma", "sigma"},   {"tau", "tau"},
        {"phi", "phi"},     {"varphi", "phi"},  {"chi", "chi"},     {"psi", "psi"},       {"omega", "omega"},
        {"Gamma", "Gamma"}, {"Delta", "Delta"}, {"Theta", "Theta"}, {"Lambda", "Lambda"}, {"Sigma", "Sigma"},
        {"Phi", "Phi"},     {"Psi", "Psi"},     {"Omega", "Omega"}};
    return m;
}

struct Names {
    std::map<std::string, PNode> bind;  // name -> Var / Par / Sym(pi)
    bool lenient = false;               // unknown names become plain symbols
    PNode resolve(const std::string& n) const {
        auto it = bind.find(n);
        if (it != bind.end()) return it->second;
        if (!lenient) throw std::runtime_error("unknown symbol: " + n);
        auto s = std::make_shared<Node>();
        s->kind = Node::Sym;
        s->name = n;
        return s;
    }
};

struct LatexExpr {
    const std::string& s;
    const Names& names;
    size_t i = 0;
    LatexExpr(const std::string& src, const Names& nm) : s(src), names(nm) {}

    void ws() {
        while (i < s.size() && std::isspace((unsigned char)s[i])) ++i;
    }
    char peek() {
        ws();
        return i < s.size() ? s[i] : '\0';
    }
    bool eat(char c) {
        ws();
        if (i < s.size() && s[i] == c) {
            ++i;
            return true;
        }
        return false;
    }
    bool starts(const char* lit) { return s.compare(i, std::strlen(lit), lit) == 0; }
    std::string command() {
        size_t j = i;
        while (j < s.size() && std::isalpha((unsigned char)s[j])) ++j;
        std::string c = s.substr(i, j - i);
        i = j;
        return c;
    }
    PNode number() {
        size_t j = i;
        while (j < s.size() && (std::isdigit((unsigned char)s[j]) || s[j] == '.')) ++j;
        if (j < s.size() && (s[j] == 'e' || s[j] == 'E')) {
            ++j;
            if (j < s.size() && (s[j] == '+' || s[j] == '-')) ++j;
            while (j < s.size() && std::isdigit((unsigned char)s[j])) ++j;
        }
        const std::string t = s.substr(i, j - i);
        double v;
        try {
            v = std::stod(t);
        } catch (...) {
            throw std::runtime_error("bad number: '" + t + "'");
        }
        i = j;
        return num(v);
    }
    PNode symbol(const std::string& n) { return names.resolve(n); }

    PNode parse() {
        PNode e = expr();
        ws();
        if (i != s.size()) throw std::runtime_error("trailing input at pos " + std::to_string(i));
        return e;
    }
    PNode expr() {
        PNode n = term();
        for (;;) {
            const char c = peek();
            if (c == '+') { eat('+'); n = binop(Node::Add, n, term()); }
            else if (c == '-') { eat('-'); n = binop(Node::Sub, n, term()); }
            else return n;
        }
    }
    bool operand_starts_here() {
        ws();
        if (i >= s.size()) return false;
        const char c = s[i];
        if (c == '(' || c == '{' || std::isdigit((unsigned char)c) || c == '.' || std::isalpha((unsigned char)c) ||
            c == '_')
            return true;
        if (c == '\\') return !(starts("\\cdot") || starts("\\right"));
        return false;
    }
    PNode term() {
        PNode n = power();
        for (;;) {
            ws();
            if (starts("\\cdot")) { i += 5; n = binop(Node::Mul, n, power()); continue; }
            const char c = peek();
            if (c == '*') { eat('*'); n = binop(Node::Mul, n, power()); }
            else if (c == '/') { eat('/'); n = binop(Node::Div, n, power()); }
            else if (operand_starts_here()) n = binop(Node::Mul, n, power());
            else return n;
        }
    }
    PNode power() {
        PNode base = unary();
        if (peek() == '^') {
            eat('^');
            return binop(Node::Pow, base, group_or_single());
        }
        return base;
    }
    PNode unary() {
        const char c = peek();
        if (c == '-') { eat('-'); return neg(unary()); }
        if (c == '+') { eat('+'); return unary(); }
        return primary();
    }
    PNode group_or_single() {
        ws();
        if (i < s.size() && s[i] == '{') {
            ++i;
            PNode e = expr();
            ws();
            if (i >= s.size() || s[i] != '}') throw std::runtime_error("expected } ");
            ++i;
            return e;
        }
        return single();
    }
    PNode single() {
        ws();
        const char c = i < s.size() ? s[i] : '\0';
        if (std::isdigit((unsigned char)c) || c == '.') return number();
        if (c == '\\') {
            ++i;
            const std::string cmd = command();
            auto g = greek().find(cmd);
            if (g != greek().end()) return symbol(g->second);
            throw std::runtime_error("unexpected latex command \\" + cmd + " as single arg");
        }
        if (std::isalpha((unsigned char)c) || c == '_') {
            size_t j = i;
            while (j < s.size() && (std::isalnum((unsigned char)s[j]) || s[j] == '_')) ++j;
            const std::string id = s.substr(i, j - i);
            i = j;
            return symbol(id);
        }
        return primary();
    }
    PNode primary() {
        ws();
        const char c = i < s.size() ? s[i] : '\0';
        if (c == '(') {
            ++i;
            PNode e = expr();
            if (!eat(')')) throw std::runtime_error("expected )");
            return e;
        }
        if (starts("\\left")) {
            i += 5;
            ws();
            if (i < s.size() && (s[i] == '(' || s[i] == '[')) ++i;
            PNode e = expr();
            ws();
            if (starts("\\right")) {
                i += 6;
                ws();
                if (i < s.size() && (s[i] == ')' || s[i] == ']')) ++i;
            }
            return e;
        }
        if (c == '{') {
            ++i;
            PNode e = expr();
            ws();
            if (i >= s.size() || s[i] != '}') throw std::runtime_error("expected }");
            ++i;
            return e;
        }
        if (c == '\\') {
            ++i;
            const std::string cmd = command();
            if (cmd == "frac") {
                PNode a = group_or_single();
                PNode b = group_or_single();
                return binop(Node::Div, a, b);
            }
            auto fn = latex_calls().find(cmd);
            if (fn != latex_calls().end()) {
                PNode exponent;
                if (peek() == '^') {
                    eat('^');
                    exponent = group_or_single();
                }
                PNode callnode = call(fn->second, {group_or_single()});
                if (exponent) return binop(Node::Pow, callnode, exponent);
                return callnode;
            }
            auto g = greek().find(cmd);
            if (g != greek().end()) return symbol(g->second);
            throw std::runtime_error("unknown latex command \\" + cmd);
        }
        if (std::isdigit((unsigned char)c) || c == '.') return number();
        if (std::isalpha((unsigned char)c) || c == '_') {
            size_t j = i;
            while (j < s.size() && (std::isalnum((unsigned char)s[j]) || s[j] == '_')) ++j;
            const std::string id = s.substr(i, j - i);
            i = j;
            if (peek() == '(') {
                if (!call_names().count(id)) throw std::runtime_error("unknown function: " + id);
                eat('(');
                std::vector<PNode> args;
                if (peek() != ')') {
                    args.push_back(expr());
                    while (peek() == ',') {
                        eat(',');
                        args.push_back(expr());
                    }
                }
                if (!eat(')')) throw std::runtime_error("expected ) after " + id);
                return call(id, args);
            }
            return symbol(id);
        }
        throw std::runtime_error(std::string("unexpected char '") + c + "' at pos " + std::to_string(i));
    }
};

}  // namespace

FuncDefs parse_func_defs(const std::string& text) {
    FuncDefs out;
    const std::string s = normalise(text);
    std::vector<std::string> lines;
    for (auto& part : split_on_double_backslash(s)) {
        std::istringstream in(part);
        std::string ln;
        while (std::getline(in, ln)) lines.push_back(ln);
    }
    for (auto& line : lines) {
        const size_t eq = line.find('=');
        if (eq == std::string::npos) continue;
        const std::string lhs = line.substr(0, eq);
        std::string rhs = line.substr(eq + 1);
        std::smatch m;
        if (!std::regex_search(lhs, m, std::regex(R"(\s*([A-Za-z]\w*)\s*\(\s*([^)]*)\s*\))"))) continue;
        FuncDef def;
        std::string cur;
        const std::string args = m[2];
        for (char c : args + ",") {
            if (c == ',') {
                const std::string t = trim(cur);
                if (!t.empty()) def.args.push_back(t);
                cur.clear();
            } else {
                cur += c;
            }
        }
        const size_t a = rhs.find_first_not_of(" \t");
        if (a != std::string::npos) rhs = rhs.substr(a);
        while (!rhs.empty() && (rhs.back() == ',' || rhs.back() == ';' || rhs.back() == '.' || rhs.back() == ' ' ||
                                rhs.back() == '\t'))
            rhs.pop_back();
        rhs = std::regex_replace(rhs, std::regex(R"(_\s*\{([A-Za-z0-9]+)\})"), "_$1");
        def.body = bars_to_fabs(rhs);
        if (!def.body.empty()) out[std::string(m[1])] = def;
    }
    if (out.empty()) throw std::runtime_error("no function definitions found (expected name(args) = body)");
    return out;
}

// System with right-hand sides kept as text until bound (see emit_scheme).
struct TextSystem {
    std::vector<std::string> vars, params, rhs;
};

static TextSystem parse_text_system(const std::string& text, const std::vector<std::string>& alphabet,
                                    bool order_as_in_system, const FuncDefs& funcs) {
    std::set<std::string> names, commands;
    for (auto& a : alphabet) {
        if (a.size() >= 2 && std::all_of(a.begin(), a.end(), [](char ch) { return std::isalpha((unsigned char)ch); }))
            commands.insert(a);
        names.insert(a);
    }
    const std::string s = normalise(text);
    std::vector<std::string> rows;
    for (auto& r : split_on_double_backslash(s))
        if (r.find_first_not_of(" \t\n\r") != std::string::npos) rows.push_back(r);
    if (rows.empty()) throw std::runtime_error("no equations found in OCR output");
    TextSystem sys;
    for (auto& row : rows) {
        const std::string eqn = strip_wrapping(row);
        const size_t eq = eqn.find('=');
        if (eq == std::string::npos) {
            if (std::none_of(eqn.begin(), eqn.end(), [](char ch) { return std::isalpha((unsigned char)ch); }))
                continue;
            throw std::runtime_error("equation without '=' (LHS with derivative required): " + eqn);
        }
        const std::string lhs = strip_wrapping(eqn.substr(0, eq));
        const std::string rhs = strip_wrapping(eqn.substr(eq + 1));
        const std::string v = lhs_variable(lhs);
        if (v.empty()) throw std::runtime_error("cannot detect state variable in LHS: '" + lhs + "'");
        sys.vars.push_back(v);
        std::string r2 = explicit_products(inline_functions(rhs, funcs), names, commands);
        const size_t a = r2.find_first_not_of(" \t");
        if (a != std::string::npos) r2 = r2.substr(a);
        sys.rhs.push_back(r2);
    }
    const std::set<std::string> varset(sys.vars.begin(), sys.vars.end());
    std::set<std::string> allowed;
    for (auto& a : alphabet)
        if (!varset.count(a) && a != "pi") allowed.insert(a);
    if (!order_as_in_system) {
        for (auto& a : alphabet)
            if (allowed.count(a)) sys.params.push_back(a);
    } else {
        std::set<std::string> seen;
        for (const auto& rhs : sys.rhs) {
            size_t i = 0;
            while (i < rhs.size()) {
                std::string tok;
                if (rhs[i] == '\\') {
                    size_t j = i + 1;
                    while (j < rhs.size() && std::isalpha((unsigned char)rhs[j])) ++j;
                    tok = rhs.substr(i + 1, j - i - 1);
                    i = j;
                } else if (std::isalpha((unsigned char)rhs[i]) || rhs[i] == '_') {
                    size_t j = i;
                    while (j < rhs.size() && (std::isalnum((unsigned char)rhs[j]) || rhs[j] == '_')) ++j;
                    tok = rhs.substr(i, j - i);
                    i = j;
                } else {
                    ++i;
                    continue;
                }
                if (allowed.count(tok) && !seen.count(tok)) {
                    seen.insert(tok);
                    sys.params.push_back(tok);
                }
            }
        }
        for (auto& a : alphabet)
            if (allowed.count(a) && !seen.count(a)) {
                sys.params.push_back(a);
                seen.insert(a);
            }
    }
    return sys;
}

static std::vector<PNode> bind_rhs(const TextSystem& t, bool lenient) {
    Names nm;
    nm.lenient = lenient;
    for (size_t i = 0; i < t.vars.size(); ++i) nm.bind[t.vars[i]] = var((int)i);
    for (size_t j = 0; j < t.params.size(); ++j) nm.bind[t.params[j]] = par(1 + (int)j);
    {
        auto n = std::make_shared<Node>();
        n->kind = Node::Sym;
        n->name = "pi";
        nm.bind["pi"] = n;
    }
    std::vector<PNode> out;
    for (auto& r : t.rhs) {
        LatexExpr p(r, nm);
        out.push_back(p.parse());
    }
    return out;
}

System parse_system(const std::string& text, const std::vector<std::string>& alphabet, bool order_as_in_system,
                    const FuncDefs& funcs) {
    TextSystem t = parse_text_system(text, alphabet, order_as_in_system, funcs);
    System s;
    s.vars = t.vars;
    s.params = t.params;
    try {
        s.rhs = bind_rhs(t, false);
    } catch (const std::runtime_error& e) {
        const std::string msg = e.what();
        if (msg.rfind("unknown symbol: ", 0) != 0) throw;
        s.bind_error = msg;
        s.rhs = bind_rhs(t, true);
    }
    return s;
}

std::string emit_scheme(const System& s, Scheme sc) {
    if (sc == Scheme::CD) return emit_cd(s);
    if (!s.bind_error.empty()) throw std::runtime_error(s.bind_error);
    const int N = (int)s.vars.size();
    if ((int)s.rhs.size() != N) throw std::runtime_error("vars/rhs size mismatch");
    std::ostringstream o;
    auto f = [&](const std::string& st) {
        std::vector<std::string> v;
        for (auto& r : s.rhs) v.push_back(emit_expr(r, st));
        return v;
    };
    switch (sc) {
        case Scheme::Euler: {
            auto k = f("X");
            o << "    numb X1[" << N << "];\n    int i;\n";
            for (int i = 0; i < N; ++i) o << "    X1[" << i << "] = X[" << i << "] + h * (" << k[i] << ");\n";
            o << "    for (i = 0; i < " << N << "; i++)\n        X[i] = X1[i];\n";
            break;
        }
        case Scheme::EulerCromer: {
            auto k = f("X");
            for (int i = 0; i < N; ++i) o << "    X[" << i << "] = X[" << i << "] + h * (" << k[i] << ");\n";
            break;
        }
        case Scheme::ExplicitMidpoint: {
            auto k0 = f("X"), k1 = f("X1");
            o << "    numb X1[" << N << "];\n";
            for (int i = 0; i < N; ++i) o << "    X1[" << i << "] = X[" << i << "] + 0.5 * h * (" << k0[i] << ");\n";
            for (int i = 0; i < N; ++i) o << "    X[" << i << "] = X[" << i << "] + h * (" << k1[i] << ");\n";
            break;
        }
        case Scheme::RK4: {
            auto k = f("X1");
            o << "    numb X1[" << N << "];\n    numb k[" << N << "][4];\n    int N = " << N << ";\n    int i, j;\n";
            o << "    for (i = 0; i < N; i++) {\n        X1[i] = X[i];\n    }\n";
            o << "    for (j = 0; j < 4; j++) {\n";
            for (int i = 0; i < N; ++i) o << "        k[" << i << "][j] = (" << k[i] << ");\n";
            o << "        if (j == 3) {\n            for (i = 0; i < N; i++) {\n            X[i] = X[i] + h * (k[i][0] + "
                 "2 * k[i][1] + 2 * k[i][2] + k[i][3]) / 6;\n            }\n        }\n";
            o << "        else if (j == 2) {\n            for (i = 0; i < N; i++) {\n            X1[i] = X[i] + h * "
                 "k[i][j];\n            }\n        }\n";
            o << "        else {\n            for (i = 0; i < N; i++) {\n                X1[i] = X[i] + 0.5 * h * "
                 "k[i][j];\n            }\n        }\n    }\n";
            break;
        }
        case Scheme::DOPRI78: {
            // Dormand-Prince 8(7), 13 stages (Prince & Dormand 1981): the stage matrix and
            // the two weight rows as the reference body prints them (12 to 13 significant
            // digits), then the 8th-order update; the 7th-order solution z is computed and
            // left unused, as in the reference body (codegen.cpp:611-675).
            static const char* const kM[13] = {
                "0,0,0,0,0,0,0,0,0,0,0,0",
                "0.05555555555556,0,0,0,0,0,0,0,0,0,0,0",
                "0.02083333333333,0.0625,0,0,0,0,0,0,0,0,0,0",
                "0.03125,0,0.09375,0,0,0,0,0,0,0,0,0",
                "0.3125,0,-1.171875,1.171875,0,0,0,0,0,0,0,0",
                "0.0375,0,0,0.1875,0.15,0,0,0,0,0,0,0",
                "0.04791013711111,0,0,0.1122487127778,-0.02550567377778,0.01284682388889,0,0,0,0,0,0",
                "0.01691798978729,0,0,0.387848278486,0.0359773698515,0.1969702142157,-0.1727138523405,0,0,0,0,0",
                "0.06909575335919,0,0,-0.6342479767289,-0.1611975752246,0.1386503094588,0.9409286140358,"
                "0.2116363264819,0,0,0,0",
                "0.183556996839,0,0,-2.468768084316,-0.2912868878163,-0.02647302023312,2.847838764193,"
                "0.2813873314699,0.1237448998633,0,0,0",
                "-1.215424817396,0,0,16.67260866595,0.9157418284168,-6.056605804357,-16.00357359416,"
                "14.8493030863,-13.37157573529,5.13418264818,0,0",
                "0.2588609164383,0,0,-4.774485785489,-0.435093013777,-3.049483332072,5.577920039936,"
                "6.155831589861,-5.062104586737,2.193926173181,0.1346279986593,0",
                "0.8224275996265,0,0,-11.65867325728,-0.7576221166909,0.7139735881596,12.07577498689,"
                "-2.12765911392,1.990166207049,-0.234286471544,0.1758985777079,0"};
            static const char* const kB[2] = {
                "0.04174749114153,0,0,0,0,-0.05545232861124,0.2393128072012,0.7035106694034,-0.7597596138145,"
                "0.6605630309223,0.1581874825101,-0.2381095387529,0.25",
                "0.02955321367635,0,0,0,0,-0.8286062764878,0.3112409000511,2.4673451906,-2.546941651842,"
                "1.443548583677,0.07941559588113,0.04444444444444,0"};
            auto k = f("X1");
            o << "    static const numb M[13][12] = {\n";
            for (int r = 0; r < 13; ++r) o << "        {" << kM[r] << "}" << (r < 12 ? ",\n" : "\n");
            o << "    };\n    static const numb B[2][13] = {\n";
            for (int r = 0; r < 2; ++r) o << "        {" << kB[r] << "}" << (r < 1 ? ",\n" : "\n");
            o << "    };\n";
            for (const char* arr : {"X1", "X2", "y", "z"}) o << "    numb " << arr << "[" << N << "];\n";
            o << "    numb k[" << N << "][13];\n    int N = " << N << ";\n    int i, j, l;\n";
            o << "    for (i = 0; i < N; ++i) X1[i] = X[i];\n    for (i = 0; i < 13; ++i) {\n";
            for (int v = 0; v < N; ++v) o << "        k[" << v << "][i] = (" << k[v] << ");\n";
            o << "        if (i != 12) {\n            for (l = 0; l < N; ++l) X2[l] = 0;\n"
                 "            for (j = 0; j < i + 1; ++j)\n                for (l = 0; l < N; ++l)\n"
                 "                    X2[l] += M[i + 1][j] * k[l][j];\n            for (l = 0; l < N; ++l)\n"
                 "                X1[l] = X[l] + h * X2[l];\n        }\n    }\n";
            for (int w = 0; w < 2; ++w)
                o << "    for (l = 0; l < N; ++l) X2[l] = 0;\n    for (i = 0; i < 13; ++i)\n"
                     "        for (l = 0; l < N; ++l)\n            X2[l] += B["
                  << w << "][i] * k[l][i];\n    for (l = 0; l < N; ++l)\n        " << (w ? "z" : "y")
                  << "[l] = X[l] + h * X2[l];\n";
            o << "    (void)z[0];\n    for (l = 0; l < N; ++l) X[l] = y[l];\n";
            break;
        }
        case Scheme::CD:
            break;  // emit_cd above
    }
    return o.str();
}

}  // namespace fe
}  // namespace ucb
