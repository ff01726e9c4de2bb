// C ABI of the text front-end (system text -> step body).
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/ucb.h"
#include "frontend.h"

namespace {

void copy_out(char* dst, int len, const std::string& s) {
    if (!dst || len <= 0) return;
    std::snprintf(dst, (size_t)len, "%s", s.c_str());
}

std::string join(const std::vector<std::string>& v) {
    std::string s;
    for (size_t i = 0; i < v.size(); ++i) s += (i ? "," : "") + v[i];
    return s;
}

}  // namespace

extern "C" UCB_API int ucb_codegen(const char* text, const char* alphabet, int order_as_in_system,
                                   const char* func_defs, int scheme, char* out, int out_len, char* vars_out,
                                   int vars_len, char* params_out, int params_len) {
    using namespace ucb::fe;
    try {
        if (!text || !alphabet) throw std::runtime_error("text and alphabet are required");
        std::vector<std::string> alpha;
        std::string cur;
        for (const char* p = alphabet;; ++p) {
            const char c = *p;
            if (c == ',' || c == ' ' || c == '\t' || c == '\n' || c == ';' || c == '\0') {
                if (!cur.empty()) alpha.push_back(cur);
                cur.clear();
                if (!c) break;
            } else {
                cur += c;
            }
        }
        if (alpha.empty()) throw std::runtime_error("alphabet is empty");
        FuncDefs funcs;
        if (func_defs && *func_defs) funcs = parse_func_defs(func_defs);
        System s = parse_system(text, alpha, order_as_in_system != 0, funcs);
        Scheme sc;
        switch (scheme) {
            case UCB_SCHEME_EULER: sc = Scheme::Euler; break;
            case UCB_SCHEME_EULER_CROMER: sc = Scheme::EulerCromer; break;
            case UCB_SCHEME_MIDPOINT: sc = Scheme::ExplicitMidpoint; break;
            case UCB_SCHEME_RK4: sc = Scheme::RK4; break;
            case UCB_SCHEME_DOPRI78: sc = Scheme::DOPRI78; break;
            case UCB_SCHEME_CD: sc = Scheme::CD; break;
            default: throw std::runtime_error("scheme not generated by this front-end");
        }
        const std::string body = emit_scheme(s, sc);
        if ((int)body.size() + 1 > out_len) throw std::runtime_error("output buffer too small");
        copy_out(out, out_len, body);
        copy_out(vars_out, vars_len, join(s.vars));
        copy_out(params_out, params_len, join(s.params));
        return UCB_OK;
    } catch (const std::exception& e) {
        copy_out(out, out_len, e.what());
        return UCB_E_INVALID;
    }
}
