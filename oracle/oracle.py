"""ORACLE (test infrastructure): ctypes wrapper over oracle/liboracle.so.

The CPU restatement of the reference hot path lives in oracle/krs_oracle.cpp; every
function there cites the reference file:line it follows. Only tests/, the smoke check
in __graft_entry__.py and bench.py's CPU-baseline leg may import this module, and only
as the checker / the timed CPU baseline. The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"

_lib = None


def build() -> None:
    """Compile liboracle.so (g++, OpenMP)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = C.CDLL(str(LIB_PATH))
        L.orc_last_error.restype = C.c_char_p
        L.orc_krs_compile.restype = C.c_void_p
        L.orc_krs_compile.argtypes = [C.c_char_p, C.c_int, C.c_int]
        L.orc_krs_free.argtypes = [C.c_void_p]
        L.orc_loop.restype = C.c_int
        L.orc_loop.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_longlong, C.c_int,
                               C.c_int, C.c_double, C.c_void_p]
        L.orc_steps.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_longlong]
        L.orc_axis_values.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, C.c_void_p]
        L.orc_rng_uniforms.argtypes = [C.c_ulonglong, C.c_int, C.c_void_p]
        grid_args = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int,
                     C.c_void_p, C.c_int, C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_double,
                     C.c_double, C.c_double, C.c_void_p, C.c_longlong, C.c_void_p, C.c_void_p, C.c_int]
        L.orc_lle2d.restype = C.c_int
        L.orc_lle2d.argtypes = grid_args
        L.orc_ls2d.restype = C.c_int
        L.orc_ls2d.argtypes = grid_args
        L.orc_bif1d.restype = C.c_int
        L.orc_bif1d.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int,
                                C.c_void_p, C.c_int, C.c_void_p, C.c_double, C.c_double, C.c_double,
                                C.c_int, C.c_int, C.c_double, C.c_int, C.c_void_p, C.c_longlong,
                                C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        L.orc_bif2d.restype = C.c_int
        L.orc_bif2d.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int,
                                C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_double, C.c_double, C.c_double,
                                C.c_int, C.c_int, C.c_double, C.c_double, C.c_void_p, C.c_longlong, C.c_void_p,
                                C.c_void_p, C.c_int]
        L.orc_rhs_compile.restype = C.c_void_p
        L.orc_rhs_compile.argtypes = [C.c_char_p, C.c_int, C.c_int]
        L.orc_ls2d_dp5.restype = C.c_int
        L.orc_ls2d_dp5.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int,
                                   C.c_void_p, C.c_int, C.c_void_p, C.c_double, C.c_double, C.c_double,
                                   C.c_double, C.c_double, C.c_int, C.c_longlong, C.c_double, C.c_void_p,
                                   C.c_longlong, C.c_void_p, C.c_void_p, C.c_int]
        L.orc_basins.restype = C.c_int
        L.orc_basins.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                 C.c_double, C.c_void_p, C.c_int, C.c_void_p, C.c_double, C.c_int, C.c_int, C.c_int,
                                 C.c_double, C.c_int, C.c_double, C.c_double, C.c_void_p, C.c_longlong, C.c_void_p,
                                 C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        L.orc_basins_ref.restype = C.c_int
        L.orc_basins_ref.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int,
                                     C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int, C.c_double,
                                     C.c_double, C.c_int, C.c_int, C.c_double, C.c_double, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_void_p, C.c_int]
        L.orc_dbscan_cells.restype = C.c_int
        L.orc_dbscan_cells.argtypes = [C.c_longlong, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_int,
                                       C.c_void_p]
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Krs:
    """A KRS step body compiled natively (krs_cpu.cpp make_source restated)."""

    def __init__(self, body: str, nx: int, numb: str = "f64"):
        self.nx = nx
        self.numb = numb
        nb = {"f64": 8, "f32": 4, "dual": 16}[numb]
        h = lib().orc_krs_compile(body.encode(), nx, nb)
        if not h:
            raise RuntimeError(lib().orc_last_error().decode())
        self.h = h

    @property
    def dtype(self):
        return np.float64 if self.numb == "f64" else np.float32

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().orc_krs_free(self.h)
        except Exception:
            pass

    def steps(self, x, a, h, n):
        x = np.array(x, dtype=self.dtype)
        a = np.array(a, dtype=self.dtype)
        lib().orc_steps(self.h, _ptr(x), _ptr(a), h, n)
        return x

    def loop(self, x, a, h, iters, pre=1, writable=0, maxv=1e6, record=False):
        x = np.array(x, dtype=self.dtype)
        a = np.array(a, dtype=self.dtype)
        data = np.zeros(max(iters, 1), dtype=self.dtype) if record else None
        flag = lib().orc_loop(self.h, _ptr(x), _ptr(a), h, iters, pre, writable, maxv, _ptr(data))
        return flag, x, data


def axis_values(n, lo, hi, log_scale=False, numb="f64"):
    out = np.zeros(n, dtype=np.float64)
    lib().orc_axis_values(8 if numb == "f64" else 4, n, lo, hi, int(log_scale), _ptr(out))
    return out


def rng_uniforms(seq, n):
    out = np.zeros(n, dtype=np.float32)
    lib().orc_rng_uniforms(seq, n, _ptr(out))
    return out


def _grid(fn, krs, g, cells, nthreads, nvals_per_cell):
    n = g["n_pts"]
    ranges = np.array(g["ranges"], dtype=np.float64)
    ic = np.array(g["ic"], dtype=np.float64)
    vals = np.array(g["values"], dtype=np.float64)
    if cells is not None:
        cells = np.ascontiguousarray(cells, dtype=np.int64)
        m = len(cells)
        values = np.zeros(m * nvals_per_cell, dtype=np.float64)
        flags = np.zeros(m, dtype=np.int32)
    else:
        m = 0
        values = np.zeros(n * n * nvals_per_cell, dtype=np.float64)
        flags = np.zeros(n * n, dtype=np.int32)
    rc = fn(krs.h, n, g["par_or_var"], g["idx"][0], g["idx"][1], _ptr(ranges), g.get("log_mask", 0),
            g.get("h_axis", -1), int(g.get("swap_xy", 0)), _ptr(ic), len(vals), _ptr(vals), g["h"],
            g["transient_time"], g["t_max"], g["NT"], g["eps"], g["max_value"], _ptr(cells), m,
            _ptr(values), _ptr(flags), nthreads)
    if rc != 0:
        raise RuntimeError(lib().orc_last_error().decode())
    return values, flags


def lle2d(krs: Krs, g: dict, cells=None, nthreads=0):
    """run_lle_2d semantics. g: kernel-level grid dict (see tests/helpers)."""
    return _grid(lib().orc_lle2d, krs, g, cells, nthreads, 1)


def ls2d(krs: Krs, g: dict, cells=None, nthreads=0):
    return _grid(lib().orc_ls2d, krs, g, cells, nthreads, krs.nx)


def bif2d(krs: Krs, g: dict, eps_dbscan: float, pre_scaller=1, writable_var=0, cells=None, nthreads=0):
    """run_bif2d semantics: per-cell period from the reference's peak dbscan (values in
    user order, -1 with flag -1 where the dbscan result is negative). g: kernel-level grid
    dict (see tests/helpers; NT / eps unused)."""
    n = g["n_pts"]
    ranges = np.array(g["ranges"], dtype=np.float64)
    ic = np.array(g["ic"], dtype=np.float64)
    vals = np.array(g["values"], dtype=np.float64)
    if cells is not None:
        cells = np.ascontiguousarray(cells, dtype=np.int64)
        m = len(cells)
    else:
        m = n * n
    values = np.zeros(m, dtype=np.float64)
    flags = np.zeros(m, dtype=np.int32)
    rc = lib().orc_bif2d(krs.h, n, g["par_or_var"], g["idx"][0], g["idx"][1], _ptr(ranges), g.get("log_mask", 0),
                         g.get("h_axis", -1), int(g.get("swap_xy", 0)), _ptr(ic), len(vals), _ptr(vals), g["h"],
                         g["transient_time"], g["t_max"], pre_scaller, writable_var, g["max_value"], eps_dbscan,
                         _ptr(cells), m if cells is not None else 0, _ptr(values), _ptr(flags), nthreads)
    if rc != 0:
        raise RuntimeError(lib().orc_last_error().decode())
    return values, flags


def basins_ref(krs: Krs, b: dict, nthreads=0):
    """run_basins semantics (reference method): (labels, avg_peaks, avg_intervals, classes),
    row-major iy*n + ix. b: n_pts, axis_x_var, axis_y_var, axis_x_lo/hi, axis_y_lo/hi, ic,
    values, h, transient_time, t_max, pre_scaller, writable_var, max_value, eps_dbscan,
    feature1, feature2, mult1, mult2."""
    n = b["n_pts"]
    ranges = np.array([b["axis_x_lo"], b["axis_x_hi"], b["axis_y_lo"], b["axis_y_hi"]], dtype=np.float64)
    ic = np.array(b["ic"], dtype=np.float64)
    vals = np.array(b["values"], dtype=np.float64)
    labels = np.zeros(n * n, dtype=np.int32)
    f1 = np.zeros(n * n)
    f2 = np.zeros(n * n)
    cls = np.zeros(n * n, dtype=np.int32)
    rc = lib().orc_basins_ref(krs.h, n, b["axis_x_var"], b["axis_y_var"], _ptr(ranges), _ptr(ic), len(vals),
                              _ptr(vals), b["h"], b["transient_time"], b["t_max"], b.get("pre_scaller", 1),
                              b.get("writable_var", 0), b["max_value"], b["eps_dbscan"], b.get("feature1", 0),
                              b.get("feature2", 1), b.get("mult1", 1.0), b.get("mult2", 1.0), _ptr(labels),
                              _ptr(f1), _ptr(f2), _ptr(cls), nthreads)
    if rc != 0:
        raise RuntimeError(lib().orc_last_error().decode())
    return labels, f1, f2, cls


def dbscan_cells(f1, f2, helpful, eps_dbscan: float, numb="f64"):
    """run_basins_recluster semantics: cluster labels of given features / classes."""
    f1 = np.ascontiguousarray(f1, dtype=np.float64)
    f2 = np.ascontiguousarray(f2, dtype=np.float64)
    helpful = np.ascontiguousarray(helpful, dtype=np.int32)
    labels = np.zeros(len(f1), dtype=np.int32)
    rc = lib().orc_dbscan_cells(len(f1), _ptr(f1), _ptr(f2), _ptr(helpful), eps_dbscan, 8 if numb == "f64" else 4,
                                _ptr(labels))
    if rc != 0:
        raise RuntimeError(lib().orc_last_error().decode())
    return labels


def bif1d(krs: Krs, b: dict, max_out=64, pts=None, nthreads=0):
    n = b["n_pts"]
    ic = np.array(b["ic"], dtype=np.float64)
    vals = np.array(b["values"], dtype=np.float64)
    if pts is not None:
        pts = np.ascontiguousarray(pts, dtype=np.int64)
        m = len(pts)
    else:
        m = n
    counts = np.zeros(m, dtype=np.int32)
    peaks = np.full(m * max_out, np.nan)
    intervals = np.full(m * max_out, np.nan)
    rc = lib().orc_bif1d(krs.h, n, b.get("sweep_kind", 0), b["sweep_index"], b["lo"], b["hi"],
                         int(b.get("log_scale", 0)), _ptr(ic), len(vals), _ptr(vals), b["h"],
                         b["transient_time"], b["t_max"], b.get("pre_scaller", 1), b.get("writable_var", 0),
                         b["max_value"], max_out, _ptr(pts), m if pts is not None else 0, _ptr(counts),
                         _ptr(peaks), _ptr(intervals), nthreads)
    if rc != 0:
        raise RuntimeError(lib().orc_last_error().decode())
    return counts, peaks.reshape(m, max_out), intervals.reshape(m, max_out)


def rhs_statements_from_rk4(body: str) -> str:
    """Right-hand-side statements recovered from a reference RK4 body: its stage lines
    `k[i][j] = (expr);` (codegen.cpp scheme_rk4) become `dX[i] = (expr);`."""
    import re
    out = []
    for m in re.finditer(r"^\s*k\[(\d+)\]\[j\] = (.*);\s*$", body, re.M):
        out.append(f"    dX[{m.group(1)}] = {m.group(2)};")
    return "\n".join(out)


class Rhs:
    """A right-hand side compiled natively twice: in double and in forward-mode duals."""

    def __init__(self, rk4_body: str, nx: int):
        self.nx = nx
        text = rhs_statements_from_rk4(rk4_body)
        self.h = lib().orc_rhs_compile(text.encode(), nx, 8)
        self.hd = lib().orc_rhs_compile(text.encode(), nx, 16)
        if not self.h or not self.hd:
            raise RuntimeError(lib().orc_last_error().decode())


def ls2d_dp5(rhs: Rhs, g: dict, *, t_end, rtol=1e-8, atol=None, h0=0.01, gs_every=10, max_steps=10**8,
             cells=None, nthreads=0):
    n = g["n_pts"]
    ranges = np.array(g["ranges"], dtype=np.float64)
    ic = np.array(g["ic"], dtype=np.float64)
    vals = np.array(g["values"], dtype=np.float64)
    if cells is not None:
        cells = np.ascontiguousarray(cells, dtype=np.int64)
        m = len(cells)
    else:
        m = n * n
    values = np.zeros(m * rhs.nx)
    flags = np.zeros(m, dtype=np.int32)
    rc = lib().orc_ls2d_dp5(rhs.h, rhs.hd, n, g["par_or_var"], g["idx"][0], g["idx"][1], _ptr(ranges),
                            g.get("log_mask", 0), _ptr(ic), len(vals), _ptr(vals), g["transient_time"], t_end, rtol,
                            atol if atol is not None else rtol, h0, gs_every, max_steps, g["max_value"],
                            _ptr(cells), m if cells is not None else 0, _ptr(values), _ptr(flags), nthreads)
    if rc != 0:
        raise RuntimeError(lib().orc_last_error().decode())
    return values.reshape(m, rhs.nx), flags


def basins(krs: Krs, b: dict, cells=None, nthreads=0):
    """Stroboscopic classification per cell: (period, canonical x, canonical y, periods)."""
    n = b["n_pts"]
    ic = np.array(b["ic"], dtype=np.float64)
    vals = np.array(b["values"], dtype=np.float64)
    if cells is not None:
        cells = np.ascontiguousarray(cells, dtype=np.int64)
        m = len(cells)
    else:
        m = n * n
    per = np.zeros(m, dtype=np.int32)
    cx = np.zeros(m)
    cy = np.zeros(m)
    it = np.zeros(m, dtype=np.int32)
    rc = lib().orc_basins(krs.h, n, b["axis_x_var"], b["axis_y_var"], b["axis_x_lo"], b["axis_x_hi"],
                          b["axis_y_lo"], b["axis_y_hi"], _ptr(ic), len(vals), _ptr(vals), b["period"],
                          b["steps_per_period"], b["max_periods"], b["match_count"], b["match_tol"],
                          b.get("phase_var", -1), b["max_value"], b.get("merge_radius", 0.0) or 1e-4, _ptr(cells),
                          m if cells is not None else 0,
                          _ptr(per), _ptr(cx), _ptr(cy), _ptr(it), nthreads)
    if rc != 0:
        raise RuntimeError(lib().orc_last_error().decode())
    return per, cx, cy, it
