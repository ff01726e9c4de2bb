// Step-body text of the CD scheme (composition "D-method"): an explicit half step of size
// h1 = h a[0] in variable order, then an implicit half step of size h2 = h (1 - a[0]) in
// reverse order, each variable solved on its own: analytically when its right-hand side is
// linear in it, by four fixed-point iterations when it is not, by an explicit update when
// it does not appear.
//
// The text is part of the exchange format between the session layer and the engine, so it
// must equal the reference's (codegen.cpp:686-754) byte for byte. The reference decides
// linearity and splits off the variable's coefficient by rewriting the plain text of each
// right-hand side (names, powers as a^b), not its expression tree, and the result carries
// the consequences of that: an integer power x^2 prints as x^2.0 in plain form and becomes
// "pow(X[0], 2).0", a product x (y - c) counts as linear in x with coefficient 1. The rules
// below restate those text rewrites; the golden fixture of the reference's own output
// (tests/golden/codegen_cases.json) pins them.
#include <regex>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "frontend.h"

namespace ucb {
namespace fe {
namespace {

// Functions whose argument list makes a variable inside it count as nonlinear.
const char* const kCallNames[] = {"abs",  "acos", "asin", "atan", "cos",  "cosh", "exp",  "fabs",
                                  "ln",   "log",  "pow",  "sin",  "sinh", "sqrt", "tan",  "tanh"};

std::string trim(const std::string& s) {
    const size_t a = s.find_first_not_of(" \t\n\r");
    if (a == std::string::npos) return "";
    const size_t b = s.find_last_not_of(" \t\n\r");
    return s.substr(a, b - a + 1);
}

// A pattern built around a name; names that do not form a valid pattern match nothing.
bool search(const std::string& text, const std::string& pattern, std::smatch* m = nullptr) {
    try {
        const std::regex re(pattern);
        return m ? std::regex_search(text, *m, re) : std::regex_search(text, re);
    } catch (const std::exception&) {
        return false;
    }
}
bool whole(const std::string& text, const std::string& pattern, std::smatch* m = nullptr) {
    try {
        const std::regex re(pattern);
        return m ? std::regex_match(text, *m, re) : std::regex_match(text, re);
    } catch (const std::exception&) {
        return false;
    }
}
void rewrite(std::string& text, const std::string& pattern, const std::string& with) {
    try {
        text = std::regex_replace(text, std::regex(pattern), with);
    } catch (const std::exception&) {
    }
}

bool mentions(const std::string& expr, const std::string& name) { return search(expr, "\\b" + name + "\\b"); }

enum class Dependence { Absent, Linear, Nonlinear };

// How a right-hand side (plain text) depends on variable v: absent; nonlinear when the
// first power of v has an integer exponent >= 2, when v * v appears, or when v sits inside
// the parentheses of a call (up to the first closing parenthesis); linear otherwise.
Dependence dependence(const std::string& expr, const std::string& v) {
    if (!mentions(expr, v)) return Dependence::Absent;
    std::smatch m;
    if (search(expr, "\\b" + v + "\\s*\\^\\s*(\\d+)", &m)) {
        try {
            if (std::stoi(m[1].str()) >= 2) return Dependence::Nonlinear;
        } catch (const std::exception&) {
        }
    }
    if (search(expr, "\\b" + v + "\\s*\\*\\s*" + v + "\\b")) return Dependence::Nonlinear;
    for (const char* fn : kCallNames)
        if (search(expr, std::string(fn) + "\\s*\\([^)]*\\b" + v + "\\b[^)]*\\)")) return Dependence::Nonlinear;
    return Dependence::Linear;
}

// Terms of a sum: cut before every '+' / '-' after the first character, except in an
// exponent (after 'e' / 'E'); each term keeps its sign.
std::vector<std::string> terms(const std::string& expr) {
    std::vector<std::string> out;
    size_t start = 0;
    for (size_t i = 1; i < expr.size(); ++i) {
        if (expr[i] != '+' && expr[i] != '-') continue;
        if (expr[i - 1] == 'e' || expr[i - 1] == 'E') continue;
        const std::string t = trim(expr.substr(start, i - start));
        if (!t.empty()) out.push_back(t);
        start = i;
    }
    if (start < expr.size()) {
        const std::string t = trim(expr.substr(start));
        if (!t.empty()) out.push_back(t);
    }
    return out;
}

// A signed term split into its sign ("+" / "-") and body.
void sign_and_body(const std::string& term, std::string& sign, std::string& body) {
    sign = "+";
    body = term;
    if (!term.empty() && (term[0] == '-' || term[0] == '+')) {
        if (term[0] == '-') sign = "-";
        body = trim(term.substr(1));
    }
}

std::string join_rest(const std::vector<std::string>& parts) {
    std::string rest;
    for (const auto& p : parts) rest += (rest.empty() ? "" : " ") + p;
    if (!rest.empty() && rest[0] == '+') rest = trim(rest.substr(1));
    return rest;
}

// rhs = sign * coef * v + rest, read off the plain text.
struct LinearSplit {
    std::string sign = "+", coef = "1", rest;
};

// Terms inside a factor's parentheses: the bare v gives the sign, every other term is
// multiplied by the outer factor into the rest.
LinearSplit split_parenthesised(const std::string& inner_in, const std::string& v, const std::string& outer) {
    std::string inner = inner_in;
    if (!inner.empty() && inner[0] != '+' && inner[0] != '-') inner = "+" + inner;
    LinearSplit r;
    r.coef = outer;
    std::vector<std::string> parts;
    for (const auto& t : terms(inner)) {
        std::string sign, body;
        sign_and_body(t, sign, body);
        if (whole(body, "^" + v + "$")) {
            r.sign = sign;
            continue;
        }
        parts.push_back((sign == "-" ? "- " : "+ ") + outer + " * " + body);
    }
    r.rest = join_rest(parts);
    return r;
}

LinearSplit linear_split(const std::string& expr_in, const std::string& v) {
    const std::string expr = trim(expr_in);
    std::smatch m;
    // (left) * (right) with v in the right factor only
    if (whole(expr, R"(^\(([^)]+)\)\s*\*\s*\(([^)]+)\)$)", &m)) {
        const std::string left = m[1].str(), right = m[2].str();
        if (mentions(right, v) && !mentions(left, v)) return split_parenthesised(right, v, "(" + left + ")");
    }
    // name * (inner) with v inside
    if (whole(expr, R"(^([a-zA-Z_]\w*)\s*\*\s*\((.+)\)$)", &m)) {
        const std::string outer = m[1].str(), inner = m[2].str();
        if (mentions(inner, v)) return split_parenthesised(inner, v, outer);
    }
    // a plain sum: the first term that is v, name * v or v * name carries v; the
    // coefficient is the name of the last such term (1 for a bare v)
    std::string sum = expr;
    if (!sum.empty() && sum[0] != '+' && sum[0] != '-') sum = "+" + sum;
    LinearSplit r;
    bool found = false;
    std::vector<std::string> parts;
    for (const auto& t : terms(sum)) {
        std::string sign, body;
        sign_and_body(t, sign, body);
        bool has = false;
        if (whole(body, "^([a-zA-Z_]\\w*)\\s*\\*\\s*" + v + "$", &m)) {
            has = true;
            r.coef = m[1].str();
        } else if (whole(body, "^" + v + "\\s*\\*\\s*([a-zA-Z_]\\w*)$", &m)) {
            has = true;
            r.coef = m[1].str();
        } else if (whole(body, "^" + v + "$")) {
            has = true;
            r.coef = "1";
        }
        if (has && !found) {
            found = true;
            r.sign = sign;
        } else {
            parts.push_back(t);
        }
    }
    r.rest = join_rest(parts);
    return r;
}

// Plain text -> C: integer powers of a variable to pow(), ln to log, variables to X[i],
// parameters to a[1 + j], in that order.
std::string to_code(const std::string& plain, const std::vector<std::string>& vars,
                    const std::vector<std::string>& params) {
    std::string code = plain;
    for (const auto& v : vars) rewrite(code, "\\b" + v + "\\s*\\^\\s*(\\d+)", "pow(" + v + ", $1)");
    rewrite(code, R"((X\[\d+\])\s*\^\s*(\d+))", "pow($1, $2)");
    rewrite(code, "\\bln\\s*\\(", "log(");
    for (size_t i = 0; i < vars.size(); ++i) rewrite(code, "\\b" + vars[i] + "\\b", "X[" + std::to_string(i) + "]");
    for (size_t j = 0; j < params.size(); ++j)
        rewrite(code, "\\b" + params[j] + "\\b", "a[" + std::to_string(1 + j) + "]");
    return code;
}

}  // namespace

std::string emit_cd(const System& s) {
    const int N = (int)s.vars.size();
    if ((int)s.rhs.size() != N) throw std::runtime_error("vars/rhs size mismatch");
    if (N < 2) throw std::runtime_error("CD method requires N >= 2");
    std::vector<std::string> plain(N);
    for (int i = 0; i < N; ++i) plain[i] = emit_plain(s.rhs[i], s.vars, s.params);
    std::ostringstream o;
    o << "    numb h1 = h * a[0];\n    numb h2 = h * (1 - a[0]);\n";
    for (int i = 0; i < N; ++i)
        o << "    X[" << i << "] = X[" << i << "] + h1 * (" << to_code(plain[i], s.vars, s.params) << ");\n";
    for (int i = N - 1; i >= 0; --i) {
        const std::string x = "X[" + std::to_string(i) + "]";
        switch (dependence(plain[i], s.vars[i])) {
            case Dependence::Absent:
                o << "    " << x << " = " << x << " + h2 * (" << to_code(plain[i], s.vars, s.params) << ");\n";
                break;
            case Dependence::Linear: {
                // v' = sign coef v + rest  ->  v = (v + h2 rest) / (1 -+ h2 coef)
                const LinearSplit e = linear_split(plain[i], s.vars[i]);
                const std::string coef = e.coef == "1" ? "1" : to_code(e.coef, s.vars, s.params);
                const std::string op = e.sign == "-" ? "+" : "-";
                const std::string denom = coef == "1" ? "(1 " + op + " h2)" : "(1 " + op + " h2 * " + coef + ")";
                if (!e.rest.empty())
                    o << "    " << x << " = (" << x << " + h2 * (" << to_code(e.rest, s.vars, s.params) << ")) / "
                      << denom << ";\n";
                else
                    o << "    " << x << " = " << x << " / " << denom << ";\n";
                break;
            }
            case Dependence::Nonlinear: {
                const std::string start = "x" + std::to_string(i) + "_cd";
                const std::string code = to_code(plain[i], s.vars, s.params);
                o << "    numb " << start << " = " << x << ";\n";
                for (int k = 0; k < 4; ++k) o << "    " << x << " = " << start << " + h2 * (" << code << ");\n";
                break;
            }
        }
    }
    return o.str();
}

}  // namespace fe
}  // namespace ucb
