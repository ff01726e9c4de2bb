"""CPU tests of the C ABI: the library loads, exports every declared symbol, validates
requests like the reference engine, and compiles its kernels for sm_100a (NVRTC needs
no GPU)."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

import ucb
from helpers import engine_request, lle2d_case

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        for m in re.finditer(r"UCB_API\s+[\w\s\*]+?\b(ucb_\w+)\s*\(", h.read_text()):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    lib = ucb.load()
    names = declared_symbols()
    assert len(names) >= 8
    out = subprocess.run(["nm", "-D", "--defined-only", str(ucb.LIB_PATH)], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = sorted(n for n in names if n not in exported)
    assert not missing, missing
    for n in names:
        getattr(lib, n)  # resolvable through dlsym
    assert lib.ucb_abi_version() == 1


@pytest.mark.parametrize("field,value,msg", [
    ("n_pts", 0, "n_pts must be > 0"),
    ("h", 0.0, "h must be > 0"),
    ("t_max", 0.0, "t_max must be > 0"),
    ("NT", 0.0, "NT must be > 0"),
    ("eps", 0.0, "eps must be > 0"),
    ("transient_time", -1.0, "transient_time must be >= 0"),
    ("param_index", 0, "param_index (axis X) out of range"),
    ("param_index_2", 4, "param_index_2 (axis Y) out of range"),
    ("amount_of_x", 33, "amountOfX out of range"),
])
def test_lle2d_validation_messages(field, value, msg):
    eng = ucb.Engine()
    req = engine_request(ucb, lle2d_case())
    setattr(req, field, value)
    with pytest.raises(ucb.UcbError) as ei:
        eng.run_lle2d(req)
    assert ei.value.code == ucb.UCB_E_INVALID
    assert msg in str(ei.value)


def test_log_scale_and_h_sweep_validation():
    eng = ucb.Engine()
    req = engine_request(ucb, lle2d_case(log_scale=True, param_lo=-1.0))
    with pytest.raises(ucb.UcbError, match="log scale requires"):
        eng.run_lle2d(req)
    req = engine_request(ucb, lle2d_case(sweep_over_h=True, sweep_over_h_2=True))
    with pytest.raises(ucb.UcbError, match="cannot both be true"):
        eng.run_lle2d(req)
    req = engine_request(ucb, lle2d_case(t_max=0.05, NT=0.1))
    with pytest.raises(ucb.UcbError, match="amountOfPointsInBlock"):
        eng.run_lle2d(req)


def test_cancel_before_start():
    eng = ucb.Engine()
    req = engine_request(ucb, lle2d_case())
    flag = C.c_int32(1)
    req.cancel = C.pointer(flag)
    with pytest.raises(ucb.UcbError) as ei:
        eng.run_lle2d(req)
    assert ei.value.code == ucb.UCB_E_CANCELLED


@pytest.mark.parametrize("prec,mode,method", [
    (ucb.PREC_F64, ucb.MODE_EXACT, ucb.LLE_AUTO),
    (ucb.PREC_F64, ucb.MODE_NATIVE, ucb.LLE_AUTO),
    (ucb.PREC_F32, ucb.MODE_NATIVE, ucb.LLE_AUTO),
    (ucb.PREC_F32, ucb.MODE_EXACT, ucb.LLE_AUTO),
    (ucb.PREC_F64, ucb.MODE_NATIVE, ucb.LLE_TANGENT),
])
def test_lle2d_kernels_compile_for_sm100a(prec, mode, method):
    req = engine_request(ucb, lle2d_case(), precision=prec, mode=mode, lle_method=method)
    note = ucb.precompile_lle2d(req)
    assert "unavailable" not in note


def test_custom_body_falls_back_to_exact_form():
    body = "    X[0] = X[0] + h * (-X[1] - X[2]);\n    X[1] = X[1] + h * (X[0] + a[1] * X[1]);\n" \
           "    X[2] = X[2] + h * (a[2] + X[2] * (X[0] - a[3]));\n"
    c = lle2d_case(body=body)
    note = ucb.precompile_lle2d(engine_request(ucb, c))
    assert "exact form" in note


def test_bad_body_reports_compile_error():
    c = lle2d_case(body="    X[0] = X[0] + undefined_symbol;\n")
    with pytest.raises(ucb.UcbError) as ei:
        ucb.precompile_lle2d(engine_request(ucb, c))
    assert ei.value.code == ucb.UCB_E_COMPILE
    assert "undefined_symbol" in str(ei.value)
