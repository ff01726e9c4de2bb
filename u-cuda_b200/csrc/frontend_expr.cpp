// Expression trees, the KRS recogniser and the native code emitters.
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <sstream>
#include <stdexcept>

#include "frontend.h"

namespace ucb {
namespace fe {

// ----------------------------------------------------------------------------- build
static std::shared_ptr<Node> mknode(Node::Kind k) {
    auto n = std::make_shared<Node>();
    n->kind = k;
    return n;
}
PNode num(double v) {
    auto n = mknode(Node::Num);
    n->num = v;
    return n;
}
PNode var(int i) {
    auto n = mknode(Node::Var);
    n->index = i;
    return n;
}
PNode par(int j) {
    auto n = mknode(Node::Par);
    n->index = j;
    return n;
}
PNode binop(Node::Kind k, PNode a, PNode b) {
    auto n = mknode(k);
    n->a = std::move(a);
    n->b = std::move(b);
    return n;
}
PNode neg(PNode a) {
    auto n = mknode(Node::Neg);
    n->a = std::move(a);
    return n;
}
PNode call(const std::string& f, std::vector<PNode> args) {
    auto n = mknode(Node::Call);
    n->name = f;
    n->args = std::move(args);
    return n;
}
static PNode sym(const std::string& s) {
    auto n = mknode(Node::Sym);
    n->name = s;
    return n;
}

// ------------------------------------------------------------------ reference text form
// Number and operator printing of the step-body text (the exchange format between the
// session layer and the engine; reproduced so that bodies compare equal as text).
static std::string fmt_number(double v) {
    if (v == (double)(long long)v) {
        const long long iv = (long long)v;
        if (iv > -1000000000000LL && iv < 1000000000000LL) return std::to_string(iv) + ".0";
    }
    char buf[64];
    for (int p = 1; p <= 17; ++p) {
        std::snprintf(buf, sizeof buf, "%.*g", p, v);
        if (std::strtod(buf, nullptr) == v) break;
    }
    std::string s(buf);
    if (s.find('.') == std::string::npos && s.find('e') == std::string::npos && s.find("inf") == std::string::npos &&
        s.find("nan") == std::string::npos)
        s += ".0";
    return s;
}

static int binding(Node::Kind k) {
    switch (k) {
        case Node::Add:
        case Node::Sub: return 1;
        case Node::Mul:
        case Node::Div: return 2;
        case Node::Neg: return 3;
        case Node::Pow: return 4;
        default: return 5;
    }
}

static void print(const PNode& n, const std::string& st, std::ostream& o);
static void print_at(const PNode& n, const std::string& st, std::ostream& o, int level) {
    const bool paren = binding(n->kind) < level;
    if (paren) o << "(";
    print(n, st, o);
    if (paren) o << ")";
}
static void print(const PNode& n, const std::string& st, std::ostream& o) {
    switch (n->kind) {
        case Node::Num: o << fmt_number(n->num); break;
        case Node::Sym: o << n->name; break;
        case Node::Var: o << st << "[" << n->index << "]"; break;
        case Node::Par: o << "a[" << n->index << "]"; break;
        case Node::Neg: o << "-"; print_at(n->a, st, o, 3); break;
        case Node::Add: print_at(n->a, st, o, 1); o << " + "; print_at(n->b, st, o, 1); break;
        case Node::Sub: print_at(n->a, st, o, 1); o << " - "; print_at(n->b, st, o, 2); break;
        case Node::Mul: print_at(n->a, st, o, 2); o << " * "; print_at(n->b, st, o, 2); break;
        case Node::Div: print_at(n->a, st, o, 2); o << " / "; print_at(n->b, st, o, 3); break;
        case Node::Pow: {
            if (n->b->kind == Node::Num) {
                const double e = n->b->num;
                const int ie = (int)e;
                if (e == (double)ie && ie >= 2 && ie <= 4) {
                    o << "(";
                    for (int k = 0; k < ie; ++k) {
                        if (k) o << " * ";
                        print_at(n->a, st, o, 2);
                    }
                    o << ")";
                    break;
                }
            }
            o << "pow(";
            print(n->a, st, o);
            o << ", ";
            print(n->b, st, o);
            o << ")";
            break;
        }
        case Node::Call:
            o << n->name << "(";
            for (size_t k = 0; k < n->args.size(); ++k) {
                if (k) o << ", ";
                print(n->args[k], st, o);
            }
            o << ")";
            break;
    }
}

std::string emit_expr(const PNode& n, const std::string& state) {
    std::ostringstream o;
    print(n, state, o);
    return o.str();
}

// Plain form: the names of variables and parameters, powers as a^b (both operands bound
// tighter than every other operator), numbers and the other operators as in the C form.
static void print_plain(const PNode& n, const std::vector<std::string>& vars, const std::vector<std::string>& pars,
                        std::ostream& o);
static void print_plain_at(const PNode& n, const std::vector<std::string>& vars, const std::vector<std::string>& pars,
                           std::ostream& o, int level) {
    const bool paren = binding(n->kind) < level;
    if (paren) o << "(";
    print_plain(n, vars, pars, o);
    if (paren) o << ")";
}
static void print_plain(const PNode& n, const std::vector<std::string>& vars, const std::vector<std::string>& pars,
                        std::ostream& o) {
    switch (n->kind) {
        case Node::Num: o << fmt_number(n->num); break;
        case Node::Sym: o << n->name; break;
        case Node::Var: o << vars.at(n->index); break;
        case Node::Par: o << pars.at(n->index - 1); break;
        case Node::Neg: o << "-"; print_plain_at(n->a, vars, pars, o, 3); break;
        case Node::Add: print_plain_at(n->a, vars, pars, o, 1); o << " + "; print_plain_at(n->b, vars, pars, o, 1); break;
        case Node::Sub: print_plain_at(n->a, vars, pars, o, 1); o << " - "; print_plain_at(n->b, vars, pars, o, 2); break;
        case Node::Mul: print_plain_at(n->a, vars, pars, o, 2); o << " * "; print_plain_at(n->b, vars, pars, o, 2); break;
        case Node::Div: print_plain_at(n->a, vars, pars, o, 2); o << " / "; print_plain_at(n->b, vars, pars, o, 3); break;
        case Node::Pow: print_plain_at(n->a, vars, pars, o, 4); o << "^"; print_plain_at(n->b, vars, pars, o, 4); break;
        case Node::Call:
            o << n->name << "(";
            for (size_t k = 0; k < n->args.size(); ++k) {
                if (k) o << ", ";
                print_plain(n->args[k], vars, pars, o);
            }
            o << ")";
            break;
    }
}

std::string emit_plain(const PNode& n, const std::vector<std::string>& vars, const std::vector<std::string>& params) {
    std::ostringstream o;
    print_plain(n, vars, params, o);
    return o.str();
}

// ------------------------------------------------------------------ C expression parser
namespace {

struct CParser {
    const std::string& s;
    std::string state;
    size_t i = 0;
    CParser(const std::string& src, const std::string& st) : s(src), state(st) {}

    void ws() {
        while (i < s.size() && std::isspace((unsigned char)s[i])) ++i;
    }
    bool eat(char c) {
        ws();
        if (i < s.size() && s[i] == c) {
            ++i;
            return true;
        }
        return false;
    }
    [[noreturn]] void bad(const std::string& what) {
        throw std::runtime_error("KRS expression: " + what + " at offset " + std::to_string(i) + " in '" + s + "'");
    }
    PNode parse() {
        PNode e = expr();
        ws();
        if (i != s.size()) bad("trailing input");
        return e;
    }
    PNode expr() {
        PNode n = term();
        for (;;) {
            ws();
            if (i < s.size() && s[i] == '+') { ++i; n = binop(Node::Add, n, term()); }
            else if (i < s.size() && s[i] == '-') { ++i; n = binop(Node::Sub, n, term()); }
            else return n;
        }
    }
    PNode term() {
        PNode n = unary();
        for (;;) {
            ws();
            if (i < s.size() && s[i] == '*') { ++i; n = binop(Node::Mul, n, unary()); }
            else if (i < s.size() && s[i] == '/') { ++i; n = binop(Node::Div, n, unary()); }
            else return n;
        }
    }
    PNode unary() {
        ws();
        if (i < s.size() && s[i] == '-') { ++i; return neg(unary()); }
        if (i < s.size() && s[i] == '+') { ++i; return unary(); }
        return primary();
    }
    int index_suffix() {
        if (!eat('[')) bad("expected [");
        ws();
        size_t j = i;
        while (j < s.size() && std::isdigit((unsigned char)s[j])) ++j;
        if (j == i) bad("expected index");
        const int v = std::atoi(s.substr(i, j - i).c_str());
        i = j;
        if (!eat(']')) bad("expected ]");
        return v;
    }
    PNode primary() {
        ws();
        if (i >= s.size()) bad("unexpected end");
        const char c = s[i];
        if (c == '(') {
            ++i;
            PNode e = expr();
            if (!eat(')')) bad("expected )");
            return e;
        }
        if (std::isdigit((unsigned char)c) || c == '.') {
            size_t j = i;
            while (j < s.size() && (std::isdigit((unsigned char)s[j]) || s[j] == '.')) ++j;
            if (j < s.size() && (s[j] == 'e' || s[j] == 'E')) {
                ++j;
                if (j < s.size() && (s[j] == '+' || s[j] == '-')) ++j;
                while (j < s.size() && std::isdigit((unsigned char)s[j])) ++j;
            }
            // C float suffix is not produced by the text front-end; reject it explicitly.
            const std::string t = s.substr(i, j - i);
            char* end = nullptr;
            const double v = std::strtod(t.c_str(), &end);
            if (!end || *end) bad("bad number '" + t + "'");
            i = j;
            return num(v);
        }
        if (std::isalpha((unsigned char)c) || c == '_') {
            size_t j = i;
            while (j < s.size() && (std::isalnum((unsigned char)s[j]) || s[j] == '_')) ++j;
            const std::string id = s.substr(i, j - i);
            i = j;
            ws();
            if (i < s.size() && s[i] == '[') {
                const int k = index_suffix();
                if (id == state) return var(k);
                if (id == "a") return par(k);
                bad("unknown array '" + id + "'");
            }
            if (i < s.size() && s[i] == '(') {
                ++i;
                std::vector<PNode> args;
                ws();
                if (!(i < s.size() && s[i] == ')')) {
                    args.push_back(expr());
                    while (eat(',')) args.push_back(expr());
                }
                if (!eat(')')) bad("expected ) after call of " + id);
                return call(id, std::move(args));
            }
            if (id == "pi" || id == "euler") return sym(id);
            bad("unknown identifier '" + id + "'");
        }
        bad(std::string("unexpected '") + c + "'");
    }
};

std::string normalize_body(const std::string& in) {
    std::string s;
    s.reserve(in.size());
    for (char c : in)
        if (c != '\r') s += c;
    // strip trailing spaces of each line and surrounding blank lines
    std::istringstream is(s);
    std::string line, out;
    std::vector<std::string> lines;
    while (std::getline(is, line)) {
        while (!line.empty() && (line.back() == ' ' || line.back() == '\t')) line.pop_back();
        lines.push_back(line);
    }
    size_t b = 0, e = lines.size();
    while (b < e && lines[b].empty()) ++b;
    while (e > b && lines[e - 1].empty()) --e;
    for (size_t k = b; k < e; ++k) out += lines[k] + "\n";
    return out;
}

}  // namespace

PNode parse_c_expr(const std::string& text, const std::string& state) {
    CParser p(text, state);
    return p.parse();
}

// RK4 template text (codegen.cpp:597-606): the exchange form of a built-in RK4 body.
static std::string rk4_text(const std::vector<std::string>& k) {
    const int N = (int)k.size();
    std::ostringstream o;
    o << "    numb X1[" << N << "];\n    numb k[" << N << "][4];\n    int N = " << N << ";\n    int i, j;\n";
    o << "    for (i = 0; i < N; i++) {\n        X1[i] = X[i];\n    }\n";
    o << "    for (j = 0; j < 4; j++) {\n";
    for (int i = 0; i < N; ++i) o << "        k[" << i << "][j] = (" << k[i] << ");\n";
    o << "        if (j == 3) {\n            for (i = 0; i < N; i++) {\n            X[i] = X[i] + h * (k[i][0] + 2 * "
         "k[i][1] + 2 * k[i][2] + k[i][3]) / 6;\n            }\n        }\n";
    o << "        else if (j == 2) {\n            for (i = 0; i < N; i++) {\n            X1[i] = X[i] + h * "
         "k[i][j];\n            }\n        }\n";
    o << "        else {\n            for (i = 0; i < N; i++) {\n                X1[i] = X[i] + 0.5 * h * "
         "k[i][j];\n            }\n        }\n    }\n";
    return o.str();
}

bool recognize_rk4(const std::string& body, int nx, Rhs& out, std::string& why) {
    const std::string nb = normalize_body(body);
    std::vector<std::string> exprs;
    std::istringstream is(nb);
    std::string line;
    int next = 0;
    while (std::getline(is, line)) {
        const std::string head = "        k[" + std::to_string(next) + "][j] = (";
        if (line.compare(0, head.size(), head) == 0 && line.size() > head.size() + 2 &&
            line.compare(line.size() - 2, 2, ");") == 0) {
            exprs.push_back(line.substr(head.size(), line.size() - head.size() - 2));
            ++next;
        }
    }
    if ((int)exprs.size() != nx) {
        why = "not the RK4 template (found " + std::to_string(exprs.size()) + " stage expressions for " +
              std::to_string(nx) + " variables)";
        return false;
    }
    if (normalize_body(rk4_text(exprs)) != nb) {
        why = "body differs from the RK4 template";
        return false;
    }
    out.nx = nx;
    out.f.clear();
    for (auto& e : exprs) {
        PNode n = parse_c_expr(e, "X1");
        out.f.push_back(n);
    }
    // indices must be in range
    std::function<void(const PNode&)> chk = [&](const PNode& n) {
        if (!n) return;
        if (n->kind == Node::Var && (n->index < 0 || n->index >= nx))
            throw std::runtime_error("X1 index out of range in KRS body");
        if (n->kind == Node::Par && (n->index < 0 || n->index >= 64))
            throw std::runtime_error("a[] index out of range in KRS body");
        chk(n->a);
        chk(n->b);
        for (auto& c : n->args) chk(c);
    };
    for (auto& f : out.f) chk(f);
    return true;
}

// ------------------------------------------------------------------ symbolic derivative
static bool is_num(const PNode& n, double v) { return n->kind == Node::Num && n->num == v; }

PNode simplify(const PNode& e) {
    if (!e) return e;
    switch (e->kind) {
        case Node::Num:
        case Node::Var:
        case Node::Par:
        case Node::Sym: return e;
        case Node::Neg: {
            PNode a = simplify(e->a);
            if (a->kind == Node::Num) return num(-a->num);
            if (a->kind == Node::Neg) return a->a;
            return neg(a);
        }
        case Node::Call: {
            std::vector<PNode> args;
            for (auto& x : e->args) args.push_back(simplify(x));
            return call(e->name, args);
        }
        default: break;
    }
    PNode a = simplify(e->a), b = simplify(e->b);
    switch (e->kind) {
        case Node::Add:
            if (is_num(a, 0)) return b;
            if (is_num(b, 0)) return a;
            return binop(Node::Add, a, b);
        case Node::Sub:
            if (is_num(b, 0)) return a;
            if (is_num(a, 0)) return simplify(neg(b));
            return binop(Node::Sub, a, b);
        case Node::Mul:
            if (is_num(a, 0) || is_num(b, 0)) return num(0);
            if (is_num(a, 1)) return b;
            if (is_num(b, 1)) return a;
            if (is_num(a, -1)) return simplify(neg(b));
            if (is_num(b, -1)) return simplify(neg(a));
            return binop(Node::Mul, a, b);
        case Node::Div:
            if (is_num(a, 0)) return num(0);
            if (is_num(b, 1)) return a;
            return binop(Node::Div, a, b);
        case Node::Pow:
            if (is_num(b, 1)) return a;
            if (is_num(b, 0)) return num(1);
            return binop(Node::Pow, a, b);
        default: return e;
    }
}

static PNode dir(const PNode& e);

static PNode dcall(const PNode& e) {
    const std::string& f = e->name;
    auto A = [&](size_t k) { return e->args.at(k); };
    if (e->args.size() == 1) {
        PNode u = A(0), du = dir(u);
        if (is_num(du, 0)) return num(0);
        auto mul = [](PNode x, PNode y) { return binop(Node::Mul, x, y); };
        auto div = [](PNode x, PNode y) { return binop(Node::Div, x, y); };
        if (f == "sin") return mul(call("cos", {u}), du);
        if (f == "cos") return neg(mul(call("sin", {u}), du));
        if (f == "tan") return mul(binop(Node::Add, num(1), mul(call("tan", {u}), call("tan", {u}))), du);
        if (f == "exp") return mul(call("exp", {u}), du);
        if (f == "log") return div(du, u);
        if (f == "log2") return div(du, mul(u, num(0.69314718055994530942)));
        if (f == "log10") return div(du, mul(u, num(2.30258509299404568402)));
        if (f == "sqrt") return div(du, mul(num(2), call("sqrt", {u})));
        if (f == "cbrt") return div(du, mul(num(3), mul(call("cbrt", {u}), call("cbrt", {u}))));
        if (f == "sinh") return mul(call("cosh", {u}), du);
        if (f == "cosh") return mul(call("sinh", {u}), du);
        if (f == "tanh") return mul(binop(Node::Sub, num(1), mul(call("tanh", {u}), call("tanh", {u}))), du);
        if (f == "asin") return div(du, call("sqrt", {binop(Node::Sub, num(1), mul(u, u))}));
        if (f == "acos") return neg(div(du, call("sqrt", {binop(Node::Sub, num(1), mul(u, u))})));
        if (f == "atan") return div(du, binop(Node::Add, num(1), mul(u, u)));
        if (f == "fabs" || f == "abs") return mul(call("copysign", {num(1), u}), du);
        if (f == "floor" || f == "ceil") return num(0);
    }
    if (e->args.size() == 2 && f == "pow") return dir(binop(Node::Pow, A(0), A(1)));
    if (e->args.size() == 2 && f == "atan2") {
        PNode y = A(0), x = A(1);
        return binop(Node::Div,
                     binop(Node::Sub, binop(Node::Mul, x, dir(y)), binop(Node::Mul, y, dir(x))),
                     binop(Node::Add, binop(Node::Mul, x, x), binop(Node::Mul, y, y)));
    }
    throw std::runtime_error("no derivative rule for function '" + f + "'");
}

static bool is_const(const PNode& n) {
    if (!n) return true;
    if (n->kind == Node::Var) return false;
    if (!is_const(n->a) || !is_const(n->b)) return false;
    for (auto& c : n->args)
        if (!is_const(c)) return false;
    return true;
}

static PNode dir(const PNode& e) {
    switch (e->kind) {
        case Node::Num:
        case Node::Par:
        case Node::Sym: return num(0);
        case Node::Var: return par(1000 + e->index);
        case Node::Neg: return neg(dir(e->a));
        case Node::Add: return binop(Node::Add, dir(e->a), dir(e->b));
        case Node::Sub: return binop(Node::Sub, dir(e->a), dir(e->b));
        case Node::Mul:
            return binop(Node::Add, binop(Node::Mul, dir(e->a), e->b), binop(Node::Mul, e->a, dir(e->b)));
        case Node::Div: {
            // (da - (a/b) db) / b
            return binop(Node::Div, binop(Node::Sub, dir(e->a), binop(Node::Mul, binop(Node::Div, e->a, e->b), dir(e->b))),
                         e->b);
        }
        case Node::Pow: {
            PNode u = e->a, v = e->b;
            if (is_const(v)) {
                // v u^(v-1) du
                PNode vm1 = (v->kind == Node::Num) ? num(v->num - 1) : binop(Node::Sub, v, num(1));
                return binop(Node::Mul, binop(Node::Mul, v, binop(Node::Pow, u, vm1)), dir(u));
            }
            // u^v (dv log u + v du / u)
            return binop(Node::Mul, e,
                         binop(Node::Add, binop(Node::Mul, dir(v), call("log", {u})),
                               binop(Node::Div, binop(Node::Mul, v, dir(u)), u)));
        }
        case Node::Call: return dcall(e);
    }
    return num(0);
}

PNode directional_derivative(const PNode& e) { return simplify(dir(e)); }

// ------------------------------------------------------------------ native emitters
namespace {

// trig_p >= 0: cos(X1[trig_p]) / sin(X1[trig_p]) are emitted as the names cph / sph.
void emit_native(const PNode& n, std::ostream& o, bool sp, int trig_p = -1) {
    if (trig_p >= 0 && n->kind == Node::Call && n->args.size() == 1 && n->args[0]->kind == Node::Var &&
        n->args[0]->index == trig_p && (n->name == "cos" || n->name == "sin")) {
        o << (n->name == "cos" ? "cph" : "sph");
        return;
    }
    switch (n->kind) {
        case Node::Num: {
            char buf[64];
            std::snprintf(buf, sizeof buf, "%.17g", n->num);
            std::string t(buf);
            if (t.find('.') == std::string::npos && t.find('e') == std::string::npos && t.find('n') == std::string::npos)
                t += ".0";
            o << "((numb)" << t << ")";
            break;
        }
        case Node::Sym: o << n->name; break;
        case Node::Var: o << "X1[" << n->index << "]"; break;
        case Node::Par:
            if (n->index >= 1000) o << "V[" << (n->index - 1000) << "]";
            else o << "a[" << n->index << "]";
            break;
        case Node::Neg: o << "(-"; emit_native(n->a, o, sp, trig_p); o << ")"; break;
        case Node::Add: o << "("; emit_native(n->a, o, sp, trig_p); o << " + "; emit_native(n->b, o, sp, trig_p); o << ")"; break;
        case Node::Sub: o << "("; emit_native(n->a, o, sp, trig_p); o << " - "; emit_native(n->b, o, sp, trig_p); o << ")"; break;
        case Node::Mul: o << "("; emit_native(n->a, o, sp, trig_p); o << " * "; emit_native(n->b, o, sp, trig_p); o << ")"; break;
        case Node::Div: o << "("; emit_native(n->a, o, sp, trig_p); o << " / "; emit_native(n->b, o, sp, trig_p); o << ")"; break;
        case Node::Pow: {
            if (n->b->kind == Node::Num) {
                const double e = n->b->num;
                const int ie = (int)e;
                if (e == (double)ie && ie >= 2 && ie <= 8) {
                    o << "(";
                    for (int k = 0; k < ie; ++k) {
                        if (k) o << " * ";
                        emit_native(n->a, o, sp, trig_p);
                    }
                    o << ")";
                    break;
                }
            }
            o << "pow(";
            emit_native(n->a, o, sp, trig_p);
            o << ", ";
            emit_native(n->b, o, sp, trig_p);
            o << ")";
            break;
        }
        case Node::Call: {
            std::string f = n->name;
            if (f == "abs") f = "fabs";
            o << f << "(";
            for (size_t k = 0; k < n->args.size(); ++k) {
                if (k) o << ", ";
                emit_native(n->args[k], o, sp, trig_p);
            }
            o << ")";
            break;
        }
    }
}

}  // namespace

std::string emit_rhs_device(const Rhs& r, bool sp) {
    std::ostringstream o;
    o << "__device__ __forceinline__ void ucb_rhs(const numb* X1, const numb* a, numb* dX) {\n";
    for (int i = 0; i < r.nx; ++i) {
        o << "    dX[" << i << "] = ";
        emit_native(r.f[i], o, sp);
        o << ";\n";
    }
    o << "}\n";
    return o.str();
}

// ------------------------------------------------------------------ packed FP32 emitter
namespace {

void emit_packed(const PNode& n, std::ostream& o) {
    auto is_mul = [](const PNode& x) { return x->kind == Node::Mul; };
    switch (n->kind) {
        case Node::Num: {
            char buf[64];
            std::snprintf(buf, sizeof buf, "%.17g", n->num);
            o << "ucb_p2((float)" << buf << ")";
            break;
        }
        case Node::Sym: o << "ucb_p2(" << n->name << ")"; break;
        case Node::Var: o << "X1[" << n->index << "]"; break;
        case Node::Par:
            if (n->index >= 1000) o << "V[" << (n->index - 1000) << "]";
            else o << "a[" << n->index << "]";
            break;
        case Node::Neg: o << "ucb_neg2("; emit_packed(n->a, o); o << ")"; break;
        case Node::Add:
            if (is_mul(n->a) || is_mul(n->b)) {
                const PNode& m = is_mul(n->a) ? n->a : n->b;
                const PNode& c = is_mul(n->a) ? n->b : n->a;
                o << "__ffma2_rn("; emit_packed(m->a, o); o << ", "; emit_packed(m->b, o); o << ", ";
                emit_packed(c, o); o << ")";
            } else {
                o << "__fadd2_rn("; emit_packed(n->a, o); o << ", "; emit_packed(n->b, o); o << ")";
            }
            break;
        case Node::Sub:
            if (is_mul(n->a)) {  // p q - c
                o << "__ffma2_rn("; emit_packed(n->a->a, o); o << ", "; emit_packed(n->a->b, o);
                o << ", ucb_neg2("; emit_packed(n->b, o); o << "))";
            } else if (is_mul(n->b)) {  // c - p q
                o << "__ffma2_rn(ucb_neg2("; emit_packed(n->b->a, o); o << "), "; emit_packed(n->b->b, o);
                o << ", "; emit_packed(n->a, o); o << ")";
            } else {
                o << "__fadd2_rn("; emit_packed(n->a, o); o << ", ucb_neg2("; emit_packed(n->b, o); o << "))";
            }
            break;
        case Node::Mul: o << "__fmul2_rn("; emit_packed(n->a, o); o << ", "; emit_packed(n->b, o); o << ")"; break;
        case Node::Div: o << "ucb_div2("; emit_packed(n->a, o); o << ", "; emit_packed(n->b, o); o << ")"; break;
        case Node::Pow: {
            if (n->b->kind == Node::Num) {
                const double e = n->b->num;
                const int ie = (int)e;
                if (e == (double)ie && ie >= 2 && ie <= 8) {
                    // left to right, as the scalar form's a * a * ... * a
                    for (int k = 1; k < ie; ++k) o << "__fmul2_rn(";
                    emit_packed(n->a, o);
                    for (int k = 1; k < ie; ++k) {
                        o << ", ";
                        emit_packed(n->a, o);
                        o << ")";
                    }
                    break;
                }
            }
            o << "ucb_call2b(powf, ";
            emit_packed(n->a, o);
            o << ", ";
            emit_packed(n->b, o);
            o << ")";
            break;
        }
        case Node::Call: {
            std::string f = n->name;
            if (f == "abs") f = "fabs";
            if (n->args.size() == 1) {
                o << "ucb_call2(" << f << ", ";
                emit_packed(n->args[0], o);
                o << ")";
            } else if (n->args.size() == 2) {
                o << "ucb_call2b(" << f << ", ";
                emit_packed(n->args[0], o);
                o << ", ";
                emit_packed(n->args[1], o);
                o << ")";
            } else {
                throw std::runtime_error("packed form: call with " + std::to_string(n->args.size()) + " arguments");
            }
            break;
        }
    }
}

}  // namespace

std::string emit_packed_device(const Rhs& r) {
    std::ostringstream o;
    o << "#define UCB_PACKED_CODE 1\n"
         "__device__ __forceinline__ float2 ucb_p2(float c) { return make_float2(c, c); }\n"
         "__device__ __forceinline__ float2 ucb_neg2(float2 x) { return make_float2(-x.x, -x.y); }\n"
         "__device__ __forceinline__ float2 ucb_div2(float2 x, float2 y) { return make_float2(x.x / y.x, x.y / y.y); }\n"
         "#define ucb_call2(ucb_fn, ucb_arg) ([&]() { const float2 ucb_t = (ucb_arg); "
         "return make_float2(ucb_fn(ucb_t.x), ucb_fn(ucb_t.y)); }())\n"
         "#define ucb_call2b(ucb_fn, ucb_arg, ucb_arg2) ([&]() { const float2 ucb_t = (ucb_arg), ucb_u = (ucb_arg2); "
         "return make_float2(ucb_fn(ucb_t.x, ucb_u.x), ucb_fn(ucb_t.y, ucb_u.y)); }())\n";
    o << "__device__ __forceinline__ void ucb_rhs2(const float2* X1, const float2* a, float2* dX) {\n";
    for (int i = 0; i < r.nx; ++i) {
        o << "    dX[" << i << "] = ";
        emit_packed(r.f[i], o);
        o << ";\n";
    }
    o << "}\n";
    o << "__device__ __forceinline__ void ucb_jvp2(const float2* X1, const float2* a, const float2* V, float2* dV) {\n";
    for (int i = 0; i < r.nx; ++i) {
        o << "    dV[" << i << "] = ";
        emit_packed(directional_derivative(r.f[i]), o);
        o << ";\n";
    }
    o << "}\n";
    return o.str();
}

static bool uses_trig_of(const PNode& n, int p) {
    if (!n) return false;
    if (n->kind == Node::Call && n->args.size() == 1 && n->args[0]->kind == Node::Var && n->args[0]->index == p &&
        (n->name == "cos" || n->name == "sin"))
        return true;
    if (uses_trig_of(n->a, p) || uses_trig_of(n->b, p)) return true;
    for (const auto& c : n->args)
        if (uses_trig_of(c, p)) return true;
    return false;
}

bool find_trig_phase(const Rhs& r, int& p, double& rate) {
    int found = -1;
    for (int i = 0; i < r.nx; ++i) {
        if (r.f[i]->kind != Node::Num) continue;
        bool used = false;
        for (const auto& f : r.f) used = used || uses_trig_of(f, i);
        if (!used) continue;
        if (found >= 0) return false;
        found = i;
    }
    if (found < 0) return false;
    p = found;
    rate = r.f[found]->num;
    return true;
}

bool find_clock(const Rhs& r, int& p, double& rate) {
    for (int i = 0; i < r.nx; ++i) {
        if (r.f[i]->kind != Node::Num || r.f[i]->num == 0.0) continue;
        p = i;
        rate = r.f[i]->num;
        return true;
    }
    return false;
}

std::string emit_rhs_trig_device(const Rhs& r, int p, bool sp) {
    std::ostringstream o;
    o << "__device__ __forceinline__ void ucb_rhs_trig(const numb* X1, const numb* a, numb* dX, numb cph, numb sph) "
         "{\n";
    for (int i = 0; i < r.nx; ++i) {
        o << "    dX[" << i << "] = ";
        emit_native(r.f[i], o, sp, p);
        o << ";\n";
    }
    o << "    (void)cph;\n    (void)sph;\n}\n";
    return o.str();
}

std::string emit_jvp_device(const Rhs& r, bool sp) {
    std::ostringstream o;
    o << "__device__ __forceinline__ void ucb_jvp(const numb* X1, const numb* a, const numb* V, numb* dV) {\n";
    for (int i = 0; i < r.nx; ++i) {
        o << "    dV[" << i << "] = ";
        emit_native(directional_derivative(r.f[i]), o, sp);
        o << ";\n";
    }
    o << "}\n";
    return o.str();
}

std::string emit_rhs_host(const Rhs& r) {
    std::ostringstream o;
    o << "#include <cmath>\nusing namespace std;\ntypedef double numb;\n"
         "static const numb pi = 3.1415926535897932384626433832795;\n"
         "static const numb euler = 2.7182818284590452353602874713527;\n"
         "extern \"C\" void ucb_rhs(const numb* X1, const numb* a, numb* dX) {\n";
    for (int i = 0; i < r.nx; ++i) {
        o << "    dX[" << i << "] = ";
        emit_native(r.f[i], o, false);
        o << ";\n";
    }
    o << "}\nextern \"C\" void ucb_jvp(const numb* X1, const numb* a, const numb* V, numb* dV) {\n";
    for (int i = 0; i < r.nx; ++i) {
        o << "    dV[" << i << "] = ";
        emit_native(directional_derivative(r.f[i]), o, false);
        o << ";\n";
    }
    o << "}\n";
    return o.str();
}

// ------------------------------------------------------------------ FLOP counts
int flops(const PNode& e) {
    if (!e) return 0;
    switch (e->kind) {
        case Node::Num:
        case Node::Var:
        case Node::Par:
        case Node::Sym: return 0;
        case Node::Neg: return flops(e->a);
        case Node::Add:
        case Node::Sub:
        case Node::Mul:
        case Node::Div: return 1 + flops(e->a) + flops(e->b);
        case Node::Pow: {
            if (e->b->kind == Node::Num) {
                const double x = e->b->num;
                const int ie = (int)x;
                if (x == (double)ie && ie >= 2 && ie <= 8) return (ie - 1) + ie * flops(e->a);
            }
            return 1 + flops(e->a) + flops(e->b);
        }
        case Node::Call: {
            int s = 1;
            for (auto& c : e->args) s += flops(c);
            return s;
        }
    }
    return 0;
}

int rhs_flops(const Rhs& r) {
    int s = 0;
    for (auto& f : r.f) s += flops(f);
    return s;
}

static int trig_calls_of(const PNode& n, int p) {
    if (!n) return 0;
    int c = (n->kind == Node::Call && n->args.size() == 1 && n->args[0]->kind == Node::Var &&
             n->args[0]->index == p && (n->name == "cos" || n->name == "sin"))
                ? 1
                : 0;
    c += trig_calls_of(n->a, p) + trig_calls_of(n->b, p);
    for (const auto& a : n->args) c += trig_calls_of(a, p);
    return c;
}

int trig_phase_calls(const Rhs& r, int p) {
    int c = 0;
    for (auto& f : r.f) c += trig_calls_of(f, p);
    return c;
}

int rk4_step_flops(const Rhs& r, int trig_phase) {
    const int trig = trig_phase >= 0 ? trig_phase_calls(r, trig_phase) : 0;
    return 4 * (rhs_flops(r) - trig) + 12 * r.nx;
}

int rk4_tangent_step_flops(const Rhs& r, int trig_phase) {
    int j = 0;
    for (auto& f : r.f) j += flops(directional_derivative(f));
    return rk4_step_flops(r, trig_phase) + 4 * j + 12 * r.nx;
}

}  // namespace fe
}  // namespace ucb
