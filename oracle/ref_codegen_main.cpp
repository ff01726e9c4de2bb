// Test infrastructure only: a tiny command-line driver around the reference's own
// front-end (sysparse.cpp `parse_system_from_latex`, codegen.cpp `codegen_scheme`),
// compiled from the reference sources where they lie by oracle/build_ref.sh.
// It is used to generate the committed golden fixtures under tests/golden/ and is
// never linked into, or called by, the product.
//
// Usage: ref_codegen <order: alphabet|system> <alphabet csv> [funcdefs-file] < equations
// Prints the parsed System and the step body of every scheme the reference emits.
#include "codegen.hpp"
#include "sysparse.hpp"

#include <fstream>
#include <iostream>
#include <iterator>
#include <sstream>
#include <string>
#include <vector>

static std::vector<std::string> split_csv(const std::string& s) {
    std::vector<std::string> out;
    std::string cur;
    for (char c : s) {
        if (c == ',' || c == ' ') {
            if (!cur.empty()) out.push_back(cur);
            cur.clear();
        } else {
            cur += c;
        }
    }
    if (!cur.empty()) out.push_back(cur);
    return out;
}

int main(int argc, char** argv) {
    if (argc < 3) {
        std::cerr << "usage: ref_codegen <alphabet|system> <alphabet csv> [funcdefs] < text\n";
        return 2;
    }
    const ParamOrder order = std::string(argv[1]) == "system" ? ParamOrder::AsInSystem
                                                               : ParamOrder::AsInAlphabet;
    const std::vector<std::string> alpha = split_csv(argv[2]);
    std::string text((std::istreambuf_iterator<char>(std::cin)), std::istreambuf_iterator<char>());
    try {
        FuncDefs funcs;
        if (argc > 3) {
            std::ifstream f(argv[3]);
            std::string ft((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
            funcs = parse_func_defs(ft);
        }
        System s = parse_system_from_latex(text, alpha, order, funcs);
        std::cout << "@VARS";
        for (auto& v : s.vars) std::cout << " " << v;
        std::cout << "\n@PARAMS";
        for (auto& p : s.params) std::cout << " " << p;
        std::cout << "\n";
        for (auto& r : s.rhs) std::cout << "@RHS " << r << "\n";
        const std::pair<const char*, Scheme> schemes[] = {
            {"Euler", Scheme::Euler}, {"Euler-Cromer", Scheme::EulerCromer},
            {"Explicit Midpoint", Scheme::ExplicitMidpoint}, {"RK4", Scheme::RK4},
            {"DOPRI78", Scheme::DOPRI78}, {"CD", Scheme::CD}};
        for (auto& sc : schemes) {
            std::cout << "@SCHEME " << sc.first << "\n";
            try {
                std::cout << codegen_scheme(s, sc.second);
            } catch (const std::exception& e) {
                std::cout << "@ERROR " << e.what() << "\n";
            }
            std::cout << "@END\n";
        }
    } catch (const std::exception& e) {
        std::cout << "@PARSE_ERROR " << e.what() << "\n";
        return 0;
    }
    return 0;
}
