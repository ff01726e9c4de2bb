"""Regenerates tests/golden/codegen_cases.json from the reference's own text front-end.

Runs oracle/_ref/ref_codegen (built by oracle/build_ref.sh from the reference's
sysparse.cpp + codegen.cpp, compiled as-is) on each case below and records the parsed
variables / parameters and the step body of every scheme. Needs the reference tree (its
U-CUDA directory, for the library presets); the committed JSON is what the tests read.

    python tests/golden/make_golden.py <reference U-CUDA directory>   (or UCB_REFERENCE_DIR)
"""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
REF_BIN = ROOT / "oracle" / "_ref" / "ref_codegen"
LIB = None  # <reference U-CUDA directory>/library_template, set by main()

# (name, text, alphabet, order, funcdefs)
CASES = [
    ("lorenz_plain", r"\dot{x} = \sigma(y-x) \\ \dot{y} = x(\rho - z) - y \\ \dot{z} = x y - \beta z",
     "x,y,z,sigma,rho,beta", "alphabet", None),
    ("rossler_config", r"\dot{x} = -y-z \\ \dot{y} = x + a y \\ \dot{z} = b + z(x-c)", "x,y,z,a,b,c", "alphabet", None),
    ("hyper_rossler", r"\dot{x} = -y-z \\ \dot{y} = x + a y + w \\ \dot{z} = 3 + x z \\ \dot{w} = -0.5 z + d w",
     "x,y,z,w,a,d", "alphabet", None),
    ("duffing_forced", r"\dot{x} = v \\ \dot{v} = -0.15 v + x - x^{3} + 0.3\cos(s) \\ \dot{s} = 1",
     "x,v,s", "alphabet", None),
    ("duffing_t_fails", r"\dot{x} = v \\ \dot{v} = -0.15 v + x - x^{3} + 0.3\cos(t) \\ \dot{t} = 1",
     "x,v,t", "alphabet", None),
    ("hyper_rossler_swept", r"\dot{x} = -y-z \\ \dot{y} = x + p y + w \\ \dot{z} = 3 + x z \\ \dot{w} = -0.5 z + q w",
     "x,y,z,w,p,q", "alphabet", None),
    ("chen_config", r"\dot{x} = a(y-x) \\ \dot{y} = (c-a)x - x z + c y \\ \dot{z} = x y - b z", "x,y,z,a,b,c",
     "alphabet", None),
    ("frac_and_powers", r"\frac{dx}{dt} = \frac{x^{2}}{1+y^{4}} - \sqrt{z} \\ \frac{dy}{dt} = x^{5} - 2.5e-3 y \\ "
     r"\frac{dz}{dt} = \sin(x)\cos(y) + \exp{-z}", "x,y,z", "alphabet", None),
    ("frac_powers_ok", r"\frac{dx}{dt} = \frac{x^{2}}{1+y^{4}} - \sqrt{z} \\ \frac{dy}{dt} = x^{5} - 0.0025 y \\ "
     r"\frac{dz}{dt} = \sin(x)\cos(y) + \exp{-z} + \tanh{x y}", "x,y,z", "alphabet", None),
    ("prime_and_order", r"x' = k y - m x \\ y' = -x + m \\", "x,y,m,k", "system", None),
    ("abs_and_greek", r"\dot{\theta} = \omega \\ \dot{\omega} = -\gamma \omega - |\theta| + \alpha \sin(\theta)",
     "theta,omega,gamma,alpha", "alphabet", None),
    ("dxdt_slash", r"dx/dt = y \cdot x - 8/3 \\ dy/dt = -x \times y + \pi", "x,y", "alphabet", None),
    ("aux_funcs", r"\dot{x} = \alpha (y - x - h(x)) \\ \dot{y} = x - y + z \\ \dot{z} = -\beta y",
     "x,y,z,alpha,beta,m0,m1", "alphabet", "h(x) = m1*x + 0.5*(m0-m1)*(|x+1| - |x-1|)"),
    ("left_right", r"\dot{x} = \left( y - x \right) a \\ \dot{y} = x \left( b - z \right) - y \\ \dot{z} = x y - c z",
     "x,y,z,a,b,c", "alphabet", None),
    ("unary_and_nums", r"\dot{x} = -(-x) + 0 . 5 y^{2} - 1e3 \\ \dot{y} = -x^{-1} + 10 - 2^{x}", "x,y", "alphabet", None),
]


def library_cases():
    out = []
    for d in sorted(LIB.iterdir()):
        rec = json.loads((d / "system.json").read_text())
        text = rec.get("latex_text") or rec.get("plain_text")
        order = "system" if rec.get("param_order") == "AsInSystem" else "alphabet"
        funcs = rec.get("func_defs_text") if rec.get("use_aux_funcs") else None
        out.append(("library_" + d.name, text, rec["alphabet_text"], order, funcs))
    return out


def run_case(text, alphabet, order, funcs):
    args = [str(REF_BIN), order, alphabet]
    tmp = None
    if funcs:
        tmp = ROOT / "_work" / "funcs.txt"
        tmp.parent.mkdir(exist_ok=True)
        tmp.write_text(funcs)
        args.append(str(tmp))
    out = subprocess.run(args, input=text.encode(), capture_output=True, check=True).stdout.decode()
    res = {"vars": [], "params": [], "schemes": {}, "error": None}
    cur = None
    buf = []
    for line in out.splitlines(keepends=True):
        if line.startswith("@PARSE_ERROR"):
            res["error"] = line[len("@PARSE_ERROR "):].strip()
        elif line.startswith("@VARS"):
            res["vars"] = line.split()[1:]
        elif line.startswith("@PARAMS"):
            res["params"] = line.split()[1:]
        elif line.startswith("@RHS"):
            pass
        elif line.startswith("@SCHEME "):
            cur = line[len("@SCHEME "):].strip()
            buf = []
        elif line.startswith("@END"):
            body = "".join(buf)
            res["schemes"][cur] = body
            cur = None
        elif line.startswith("@ERROR ") and cur is not None:
            buf.append(line)
        elif cur is not None:
            buf.append(line)
    return res


def main():
    global LIB
    import os
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("UCB_REFERENCE_DIR", "")
    if not ref or not (Path(ref) / "library_template").is_dir():
        sys.exit("usage: make_golden.py <reference U-CUDA directory> (or UCB_REFERENCE_DIR)")
    LIB = Path(ref) / "library_template"
    if not REF_BIN.exists():
        sys.exit("oracle/_ref/ref_codegen missing: run oracle/build_ref.sh <reference U-CUDA directory> first")
    cases = []
    for name, text, alpha, order, funcs in CASES + library_cases():
        r = run_case(text, alpha, order, funcs)
        cases.append({"name": name, "text": text, "alphabet": alpha, "order": order, "funcs": funcs, **r})
    out = Path(__file__).with_name("codegen_cases.json")
    out.write_text(json.dumps({"generator": "oracle/_ref/ref_codegen (reference sysparse.cpp + codegen.cpp)",
                               "cases": cases}, indent=1))
    print(f"wrote {out} ({len(cases)} cases)")


if __name__ == "__main__":
    main()
