// Text front-end of the engine.
//
// 1. System text -> System -> step body ("KRS"), the role of the reference's
//    sysparse.cpp (parse_system_from_latex, :287-393) and codegen.cpp (codegen_scheme,
//    :951-961). The emitted step bodies are byte-identical to the reference's for the
//    schemes implemented here (Euler, Euler-Cromer, Explicit Midpoint, RK4, DOPRI78),
//    because sessions, stored custom schemes and the engine's own recogniser exchange
//    them as text.
// 2. Step body -> right-hand side: recognises the codegen RK4 template in a KRS body and
//    recovers the right-hand-side expressions as an expression tree, from which the
//    native FMA-ordered integrator code, the tangent-linear product J(x) v and the
//    algorithmic FLOP count are generated.
#pragma once

#include <map>
#include <memory>
#include <string>
#include <vector>

namespace ucb {
namespace fe {

// ------------------------------------------------------------------ expression tree
struct Node;
using PNode = std::shared_ptr<const Node>;

struct Node {
    enum Kind { Num, Sym, Var, Par, Call, Add, Sub, Mul, Div, Pow, Neg } kind;
    double num = 0;          // Num
    std::string name;        // Sym (symbolic name before binding), Call (function)
    int index = 0;           // Var: X[index]; Par: a[index]
    PNode a, b;              // operands
    std::vector<PNode> args; // Call
};

PNode num(double v);
PNode var(int i);
PNode par(int j);
PNode binop(Node::Kind k, PNode a, PNode b);
PNode neg(PNode a);
PNode call(const std::string& f, std::vector<PNode> args);

// ------------------------------------------------------------------ system text
struct System {
    std::vector<std::string> vars;    // state variables -> X[0..N-1]
    std::vector<std::string> params;  // parameters -> a[1..M] (a[0] reserved)
    std::vector<PNode> rhs;           // bound right-hand sides (Var / Par / Num / pi)
    // A name that is neither a variable, a parameter nor pi fails every scheme that binds
    // names (the message is kept here and rhs holds it as a plain symbol); the CD scheme
    // works on the plain text and passes it through, as the reference does.
    std::string bind_error;
};

struct FuncDef {
    std::vector<std::string> args;
    std::string body;
};
using FuncDefs = std::map<std::string, FuncDef>;

enum class Scheme { Euler, EulerCromer, ExplicitMidpoint, RK4, DOPRI78, CD };

// Parses a multi-line LaTeX (or plain-syntax) system with the given alphabet. Throws
// std::runtime_error with a message on malformed input.
System parse_system(const std::string& text, const std::vector<std::string>& alphabet,
                    bool order_as_in_system = false, const FuncDefs& funcs = {});
FuncDefs parse_func_defs(const std::string& text);

// Step body of a scheme, in the reference's text form.
std::string emit_scheme(const System& s, Scheme sc);
// The CD scheme's body (frontend_cd.cpp).
std::string emit_cd(const System& s);
// C expression of one right-hand side over `state` (e.g. "X1") and a[].
std::string emit_expr(const PNode& n, const std::string& state);
// Plain text of an expression: variable / parameter names, powers printed as a^b.
std::string emit_plain(const PNode& n, const std::vector<std::string>& vars, const std::vector<std::string>& params);

// ------------------------------------------------------------------ recognition
struct Rhs {
    int nx = 0;
    std::vector<PNode> f;  // dX_i/dt over Var(X1[k]) and Par(a[j])
};

// Recognises a step body produced by the RK4 template (codegen.cpp:597-606 text form).
// Returns false (with a reason) for any other body.
bool recognize_rk4(const std::string& body, int nx, Rhs& out, std::string& why);

// Parses one C expression of a KRS body (numbers, X1[k] / X[k], a[k], pi, euler,
// calls, + - * /, unary minus, parentheses).
PNode parse_c_expr(const std::string& text, const std::string& state);

// Native device code.
//   ucb_rhs(const numb* X1, const numb* a, numb* dX)
//   ucb_jvp(const numb* X1, const numb* a, const numb* V, numb* dV)   (dV = J(X1) V)
std::string emit_rhs_device(const Rhs& r, bool single_precision);
std::string emit_jvp_device(const Rhs& r, bool single_precision);
// Packed FP32 forms for two cells at once (sm_100 FFMA2 / FADD2 / FMUL2 on float2):
// ucb_rhs2(X1, a, dX) and ucb_jvp2(X1, a, V, dV) over float2, every a * b + c fused.
std::string emit_packed_device(const Rhs& r);
// A forcing phase: a variable p whose right-hand side is a constant `rate` (so it advances
// by rate * h per step) and whose sin / cos appear in the system. False if there is none
// (or more than one).
bool find_trig_phase(const Rhs& r, int& p, double& rate);
// A clock: the first variable p whose right-hand side is a nonzero constant `rate` (time
// itself, or a forcing phase). False if there is none.
bool find_clock(const Rhs& r, int& p, double& rate);
// ucb_rhs_trig(X1, a, dX, cph, sph): ucb_rhs with cos(X1[p]) / sin(X1[p]) taken from the
// arguments (the forcing evaluated by the caller, e.g. from a table of the stage phases).
std::string emit_rhs_trig_device(const Rhs& r, int p, bool single_precision);
// Host C++ source of the same two functions for numb = double (used by the CPU tools).
std::string emit_rhs_host(const Rhs& r);

// Directional derivative d/ds f(x + s v) at s = 0 as an expression tree (V[k] as Par
// nodes with index 1000 + k).
PNode directional_derivative(const PNode& e);
PNode simplify(const PNode& e);

// Algorithmic FLOPs of an expression: + - * / count 1, negation 0, a call 1 plus its
// arguments, pow with a small integer exponent as the multiplications it expands to.
int flops(const PNode& e);
int rhs_flops(const Rhs& r);
// One RK4 step of the native integrator: 4 right-hand sides + 12 N updates per
// component (3 stage FMAs of 2, the combination (k1 + k4) + 2 (k2 + k3) of 4, the final
// FMA of 2). With trig_phase >= 0, the sin / cos calls of that forcing phase are not
// counted: the native kernels take them from a table or rotate one sincos per step.
int rk4_step_flops(const Rhs& r, int trig_phase = -1);
// The same for the state and its tangent vector v' = J(x) v: 4 (F_rhs + F_jvp) + 24 N.
int rk4_tangent_step_flops(const Rhs& r, int trig_phase = -1);
// sin / cos calls of variable p in one right-hand-side evaluation.
int trig_phase_calls(const Rhs& r, int p);

}  // namespace fe
}  // namespace ucb
