"""ORACLE (test infrastructure): the reference's own integrator kernels on the GPU.

oracle/build_ref_kernels.py compiles the reference's NVRTC templates unchanged into
oracle/_ref/refk_*.cubin (two builds: "stock" = the reference's compile options, "nofma"
= the same with --fmad=false); oracle/_ref/libucb_refharness.so (oracle/ref_harness.cpp)
launches them with the host logic of the reference's run_lle_2d / run_ls_2d / run_bif1d.
Only tests import this module; the product never does. Needs a GPU.
"""
from __future__ import annotations

import ctypes as C
import json
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF = HERE / "_ref"
MANIFEST = REF / "refk_manifest.json"
HARNESS = REF / "libucb_refharness.so"

_lib = None


def available() -> bool:
    return MANIFEST.exists() and HARNESS.exists()


def manifest() -> dict:
    return json.loads(MANIFEST.read_text())


def _harness():
    global _lib
    if _lib is None:
        L = C.CDLL(str(HARNESS))
        L.refh_last_error.restype = C.c_char_p
        L.refh_lle2d.restype = C.c_int
        L.refh_lle2d.argtypes = [C.c_char_p, C.c_char_p, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                 C.c_double, C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                 C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.POINTER(C.c_float)]
        L.refh_bif1d.restype = C.c_int
        L.refh_bif1d.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, C.c_int, C.c_int, C.c_double, C.c_double,
                                 C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_double, C.c_double,
                                 C.c_double, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int, C.c_void_p,
                                 C.c_void_p, C.c_void_p, C.POINTER(C.c_float)]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _module(case: str, variant: str):
    ent = manifest()["cases"][case]
    v = ent["variants"][variant]
    return ent, str(REF / v["cubin"]), v["kernels"]


def lle2d(case: str, variant: str, g: dict, ls: bool = False):
    """LLEKernelCUDA (or LSKernelCUDA with ls=True) over the kernel-level grid g (the
    dict tests/helpers.kernel_grid builds; its par_or_var must be the module's).
    Returns (values, flags, kernel_ms): values n^2 (LLE) or n^2 x N (LS) in kernel order,
    flags as run_lle_2d / run_ls_2d set them (999 / -999 -> -1, else 1)."""
    ent, cubin, kern = _module(case, variant)
    assert g["par_or_var"] == ent["par_or_var"], "grid sweep kind differs from the compiled module"
    nx = ent["amountOfX"]
    n = g["n_pts"]
    ranges = np.array(g["ranges"], dtype=np.float64)
    idx = np.array(g["idx"], dtype=np.int32)
    ic = np.array(g["ic"], dtype=np.float64)
    vals = np.array(g["values"], dtype=np.float64)
    per = nx if ls else 1
    out = np.zeros(n * n * per)
    ms = C.c_float()
    name = kern["LSKernelCUDA" if ls else "LLEKernelCUDA"]
    rc = _harness().refh_lle2d(cubin.encode(), name.encode(), int(ls), n, g["NT"], g["t_max"], g["transient_time"],
                               g["h"], g["eps"], g["max_value"], _p(ranges), _p(idx), _p(ic), nx, _p(vals), len(vals),
                               g.get("h_axis", -1), g.get("log_mask", 0), _p(out), C.byref(ms))
    if rc != 0:
        raise RuntimeError(_harness().refh_last_error().decode())
    if ls:
        out = out.reshape(n * n, nx)
        first = out[:, 0]
    else:
        first = out
    flags = np.where((first == 999.0) | (first == -999.0), -1, 1).astype(np.int32)
    return out, flags, float(ms.value)


def bif1d(case: str, variant: str, b: dict, cap: int = 64):
    """calculateDiscreteModelCUDA + peakFinderCUDA (run_bif1d, classical form). b: the
    oracle's bif1d dict (n_pts, sweep_kind 0 param / 1 IC, sweep_index, lo, hi,
    log_scale, ic, values, h, transient_time, t_max, pre_scaller, writable_var,
    max_value). Returns (counts, peaks[n, cap], intervals[n, cap], kernel_ms) with the
    reference's counts (peak count, -1 unusable) and NaN beyond each row's peaks."""
    ent, cubin, kern = _module(case, variant)
    sweep_var = b.get("sweep_kind", 0) == 1
    assert (0 if sweep_var else 1) == ent["par_or_var"], "sweep kind differs from the compiled module"
    nx = ent["amountOfX"]
    n = b["n_pts"]
    ic = np.array(b["ic"], dtype=np.float64)
    vals = np.array(b["values"], dtype=np.float64)
    counts = np.zeros(n, dtype=np.int32)
    peaks = np.zeros(n * cap)
    intervals = np.zeros(n * cap)
    ms = C.c_float()
    rc = _harness().refh_bif1d(cubin.encode(), kern["calculateDiscreteModelCUDA"].encode(),
                               kern["peakFinderCUDA"].encode(), n, int(sweep_var), b["lo"], b["hi"],
                               b["sweep_index"], _p(ic), nx, _p(vals), len(vals), b["h"], b["transient_time"],
                               b["t_max"], b.get("pre_scaller", 1), b.get("writable_var", 0), b["max_value"],
                               int(b.get("log_scale", 0)), cap, _p(counts), _p(peaks), _p(intervals), C.byref(ms))
    if rc != 0:
        raise RuntimeError(_harness().refh_last_error().decode())
    return counts, peaks.reshape(n, cap), intervals.reshape(n, cap), float(ms.value)
