"""Shared test fixtures: systems from the golden codegen fixture and request builders
that feed the same grid to the engine (C ABI) and to the oracle."""
import json
from functools import lru_cache
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"


@lru_cache(maxsize=None)
def codegen_cases():
    return {c["name"]: c for c in json.loads((GOLDEN / "codegen_cases.json").read_text())["cases"]}


def rk4_body(case_name):
    """RK4 step body produced by the reference's codegen for a golden case."""
    return codegen_cases()[case_name]["schemes"]["RK4"]


# Reference-generated RK4 bodies of the benchmark systems.
ROSSLER = "rossler_config"      # a=a[1], b=a[2], c=a[3]
LORENZ = "library_Lorenz"       # sigma=a[1], rho=a[2], beta=a[3]
CHEN = "chen_config"            # a=a[1], b=a[2], c=a[3]
HYPER_ROSSLER = "hyper_rossler_swept"  # p=a[1] (0.25), q=a[2] (0.05)
DUFFING = "duffing_forced"      # x, v, s (phase)


def lle2d_case(n=12, t_max=20.0, transient=10.0, NT=0.1, h=0.01, **kw):
    """A small Rossler LLE map over (b, c), the shape of the 1024^2 benchmark map."""
    d = dict(body=rk4_body(ROSSLER), nx=3, ic=(1.0, 1.0, 1.0), values=(0.0, 0.2, 0.2, 5.7), n_pts=n,
             param_index=2, param_index_2=3, param_lo=0.05, param_hi=2.0, param_lo_2=2.0, param_hi_2=20.0,
             h=h, transient_time=transient, t_max=t_max, NT=NT, eps=1e-4, max_value=1e6)
    d.update(kw)
    return d


def kernel_grid(c):
    """Oracle grid dict: the kernel-level mapping run_lle_2d derives from a request
    (parametric_engine.cpp:2602-2703)."""
    sv, sv2 = c.get("sweep_over_var", False), c.get("sweep_over_var_2", False)
    sh, sh2 = c.get("sweep_over_h", False), c.get("sweep_over_h_2", False)
    lo, hi, lo2, hi2 = c["param_lo"], c["param_hi"], c["param_lo_2"], c["param_hi_2"]
    lg, lg2 = c.get("log_scale", False), c.get("log_scale_2", False)
    pi, pi2 = c.get("param_index", 0), c.get("param_index_2", 0)
    vi, vi2 = c.get("var_sweep_index", 0), c.get("var_sweep_index_2", 0)
    swap = False
    h_axis = -1
    if sh or sh2:
        h_axis = 0 if sh else 1
        other_var = sv2 if sh else sv
        pov = 0 if other_var else 1
        if sh:
            idx = (0, vi2 if pov == 0 else pi2)
        else:
            idx = (vi if pov == 0 else pi, 0)
        ranges = (lo, hi, lo2, hi2)
        logm = (1 if lg else 0) | (2 if lg2 else 0)
    elif sv == sv2:
        pov = 0 if sv else 1
        idx = (vi, vi2) if sv else (pi, pi2)
        ranges = (lo, hi, lo2, hi2)
        logm = (1 if lg else 0) | (2 if lg2 else 0)
    elif sv and not sv2:
        pov = 2
        idx = (vi, pi2)
        ranges = (lo, hi, lo2, hi2)
        logm = (1 if lg else 0) | (2 if lg2 else 0)
    else:
        pov = 2
        idx = (vi2, pi)
        ranges = (lo2, hi2, lo, hi)
        swap = True
        logm = (1 if lg2 else 0) | (2 if lg else 0)
    return dict(n_pts=c["n_pts"], par_or_var=pov, idx=idx, ranges=ranges, log_mask=logm, h_axis=h_axis,
                swap_xy=swap, ic=c["ic"], values=c["values"], h=c["h"], transient_time=c["transient_time"],
                t_max=c["t_max"], NT=c["NT"], eps=c["eps"], max_value=c["max_value"])


def engine_request(ucb, c, **opt):
    kw = {k: c[k] for k in ("n_pts", "param_index", "param_index_2", "param_lo", "param_hi", "param_lo_2",
                             "param_hi_2", "h", "transient_time", "t_max", "NT", "eps", "max_value")}
    for k in ("sweep_over_var", "sweep_over_var_2", "sweep_over_h", "sweep_over_h_2", "log_scale", "log_scale_2",
              "var_sweep_index", "var_sweep_index_2"):
        if k in c:
            kw[k] = c[k]
    return ucb.Engine.lle2d_request(c["body"], c["nx"], c["ic"], c["values"], opt=ucb.options(**opt), **kw)


def lyapunov_spread(a, b):
    d = np.abs(np.asarray(a) - np.asarray(b))
    return d
