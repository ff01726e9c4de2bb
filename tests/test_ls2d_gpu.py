"""GPU parity of the Lyapunov-spectrum maps.

FIXED (the reference's LSKernelCUDA method): exact form bit-identical trajectories, so
spectra match the oracle to 1e-12 relative (log is the only difference).
DP5 (adaptive Dormand-Prince 5(4) + tangent vectors + modified Gram-Schmidt): the oracle
runs the same algorithm on the CPU with forward-mode duals for J v; step-size sequences may
part where an error estimate sits at the acceptance threshold, so agreement is checked by
tolerance: per-exponent 1e-3 on well-conditioned cells, the known Lorenz divergence
identity sum(lambda) = -(sigma + 1 + beta), and FP32 against FP64."""
import numpy as np
import pytest

import ucb
from helpers import HYPER_ROSSLER, LORENZ, engine_request, kernel_grid, lle2d_case, rk4_body
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    e = ucb.Engine(0)
    yield e
    e.close()


def hyper_case(n=6, **kw):
    d = lle2d_case(n=n, body=rk4_body(HYPER_ROSSLER), nx=4, ic=(-10.0, -6.0, 0.0, 10.0), values=(0, 0.25, 0.05),
                   param_index=1, param_index_2=2, param_lo=0.1, param_hi=0.35, param_lo_2=0.01, param_hi_2=0.1,
                   h=0.01, transient_time=5.0, t_max=10.0, NT=0.1, eps=1e-6)
    d.update(kw)
    return d


def lorenz_case(n=4, **kw):
    d = lle2d_case(n=n, body=rk4_body(LORENZ), nx=3, ic=(0.1, 0.1, 0.1), values=(0, 10.0, 28.0, 8 / 3),
                   param_index=1, param_index_2=2, param_lo=9.0, param_hi=11.0, param_lo_2=26.0, param_hi_2=30.0,
                   h=0.01, transient_time=5.0, t_max=20.0, NT=0.1, eps=1e-6)
    d.update(kw)
    return d


def ls_request(c, method, **opt):
    kw = {k: c[k] for k in ("n_pts", "param_index", "param_index_2", "param_lo", "param_hi", "param_lo_2",
                             "param_hi_2", "h", "transient_time", "t_max", "NT", "eps", "max_value")}
    extra = {k: c[k] for k in ("t_end", "rtol", "gs_every", "sweep_over_var", "sweep_over_var_2", "var_sweep_index",
                                "var_sweep_index_2") if k in c}
    return ucb.Engine.ls2d_request(c["body"], c["nx"], c["ic"], c["values"], method=method, opt=ucb.options(**opt),
                                   **extra, **kw)


@pytest.mark.parametrize("case", ["hyper", "lorenz"])
def test_fixed_exact_matches_oracle(eng, case):
    c = hyper_case() if case == "hyper" else lorenz_case()
    v, f, res = eng.run_ls2d(ls_request(c, ucb.LS_FIXED, precision=ucb.PREC_F64, mode=ucb.MODE_EXACT))
    ov, of = O.ls2d(O.Krs(c["body"], c["nx"]), kernel_grid(c))
    ov = ov.reshape(c["nx"], -1)
    np.testing.assert_array_equal(f, of)
    np.testing.assert_allclose(v, ov, rtol=1e-12, atol=1e-13)
    assert res.steps > 0


def test_fixed_fp32_tangent_lorenz_divergence_identity(eng):
    """The native FP32 form of the fixed method follows tangent vectors (FP64 Gram-Schmidt,
    norms and log sums): for Lorenz, whose divergence is the constant -(sigma + 1 + beta),
    the spectrum sums to it exactly, times (NT/h + 1)/(NT/h) for the extra step of every
    block, on every cell of a sigma sweep."""
    c = lorenz_case(n=4, t_max=50.0)
    v, f, res = eng.run_ls2d(ls_request(c, ucb.LS_FIXED, precision=ucb.PREC_F32, mode=ucb.MODE_NATIVE))
    assert (f == 1).all() and np.isfinite(v).all()
    n = c["n_pts"]
    # cells in kernel order: axis 0 (sigma, param_index 1) varies fastest
    sig = np.tile(np.linspace(c["param_lo"], c["param_hi"], n), n)
    expect = -(sig + 1 + 8 / 3) * (0.1 / 0.01 + 1) / (0.1 / 0.01)
    np.testing.assert_allclose(v.sum(axis=0), expect, atol=5e-3)
    assert (v[0] > 0.5).all()


def test_fixed_fp32_tangent_against_fp64_on_the_hyperchaotic_window(eng):
    """On the hyper-chaotic Rossler window with eps = 1e-6 (where FP32 shadow differences
    vanish), the FP32 tangent form stays finite and follows the FP64 map. Cells are chaotic,
    so single cells part after a few Lyapunov times: the spectrum sum (the time average of the
    Jacobian's trace along the trajectory) is compared per cell within 1 % at the median, and
    each exponent through its median over the map."""
    c = hyper_case(n=8, param_lo=0.24, param_hi=0.26, param_lo_2=0.045, param_hi_2=0.055, transient_time=10.0,
                   t_max=100.0)
    v64, f64, _ = eng.run_ls2d(ls_request(c, ucb.LS_FIXED, precision=ucb.PREC_F64, mode=ucb.MODE_NATIVE))
    v32, f32, _ = eng.run_ls2d(ls_request(c, ucb.LS_FIXED, precision=ucb.PREC_F32, mode=ucb.MODE_NATIVE))
    both = (f64 == 1) & (f32 == 1)
    assert both.sum() >= 0.9 * both.size
    assert np.isfinite(v32[:, both]).all()
    s32, s64 = v32[:, both].sum(axis=0), v64[:, both].sum(axis=0)
    assert np.median(np.abs(s32 / s64 - 1)) < 1e-2
    m32, m64 = np.median(v32[:, both], axis=1), np.median(v64[:, both], axis=1)
    np.testing.assert_allclose(m32[:3], m64[:3], atol=1e-2)
    assert abs(m32[3] / m64[3] - 1) < 2e-2


def test_fixed_fp32_tangent_flags_escaping_cells_like_fp64(eng):
    """On the wide hyper-chaotic window at t_max 30 about a third of the cells escape to
    max_value (47 of 144 in the oracle). The FP32 tangent form flags the same cells as the
    FP64 form, but for a few near the escape boundary, and its bounded cells are finite."""
    c = hyper_case(n=12, t_max=30.0)
    v64, f64, _ = eng.run_ls2d(ls_request(c, ucb.LS_FIXED, precision=ucb.PREC_F64, mode=ucb.MODE_NATIVE))
    v32, f32, _ = eng.run_ls2d(ls_request(c, ucb.LS_FIXED, precision=ucb.PREC_F32, mode=ucb.MODE_NATIVE))
    assert (f64 != 1).sum() >= 30
    assert (f32 == f64).mean() >= 0.95
    assert np.isfinite(v32[:, f32 == 1]).all()


def test_fixed_swap_and_min_max(eng):
    c = hyper_case(sweep_over_var_2=True, var_sweep_index_2=0, param_lo_2=-11.0, param_hi_2=-9.0)
    v, f, res = eng.run_ls2d(ls_request(c, ucb.LS_FIXED, precision=ucb.PREC_F64, mode=ucb.MODE_EXACT))
    ov, of = O.ls2d(O.Krs(c["body"], c["nx"]), kernel_grid(c))
    np.testing.assert_array_equal(f, of)
    np.testing.assert_allclose(v, ov.reshape(c["nx"], -1), rtol=1e-12, atol=1e-13)


@pytest.mark.parametrize("prec", [ucb.PREC_F64, ucb.PREC_F32])
def test_dp5_lorenz_divergence_identity(eng, prec):
    c = lorenz_case(n=2, param_lo=10.0, param_hi=10.0, param_lo_2=28.0, param_hi_2=28.0, transient_time=10.0,
                    t_end=300.0, gs_every=10)
    v, f, res = eng.run_ls2d(ls_request(c, ucb.LS_DP5, precision=prec))
    assert (f == 1).all()
    s = v.sum(axis=0)
    tol = 1e-3 if prec == ucb.PREC_F64 else 2e-2
    np.testing.assert_allclose(s, -(10 + 1 + 8 / 3), atol=tol)
    assert (np.abs(v[0] - 0.906) < 0.08).all()


# The hyperchaotic window around the classic parameters (0.25, 0.05): every cell on the
# attractor or escaping, 4th exponent -15 .. -80 (the full configuration grid also holds
# near-escape cells with exponents near -5000 that need ~1e6 tiny steps each).
WINDOW = dict(param_lo=0.24, param_hi=0.26, param_lo_2=0.045, param_hi_2=0.055)


def test_dp5_matches_oracle(eng):
    c = hyper_case(n=4, transient_time=20.0, t_end=200.0, gs_every=10, **WINDOW)
    v, f, res = eng.run_ls2d(ls_request(c, ucb.LS_DP5, precision=ucb.PREC_F64))
    g = kernel_grid(c)
    ov, of = O.ls2d_dp5(O.Rhs(c["body"], 4), g, t_end=200.0, rtol=1e-8, h0=c["h"], gs_every=10)
    np.testing.assert_array_equal(f, of)
    ov = ov.T
    # the sum of the spectrum (the time-averaged divergence) is robust to step-sequence
    # differences; individual exponents of hyperchaotic cells are finite-time samples
    np.testing.assert_allclose(v.sum(axis=0), ov.sum(axis=0), atol=5e-3)
    assert np.median(np.abs(v - ov)) < 5e-3


def test_dp5_f32_close_to_f64(eng):
    # FP32 state and tangent vectors at the FP32 tolerance (rtol 1e-5) against FP64 at the
    # same tolerance: the strongly contracting 4th exponents (-15 .. -5400 on this grid)
    # are resolved because the error norm covers the tangent vectors; the remaining
    # dependence on rtol itself is a property of the method, not of the precision.
    c = hyper_case(n=4, transient_time=20.0, t_end=100.0, gs_every=10, rtol=1e-5, **WINDOW)
    v64, f64, _ = eng.run_ls2d(ls_request(c, ucb.LS_DP5, precision=ucb.PREC_F64))
    v32, f32, _ = eng.run_ls2d(ls_request(c, ucb.LS_DP5, precision=ucb.PREC_F32))
    np.testing.assert_array_equal(f32, f64)
    ok = f64 == 1
    assert ok.sum() >= 3
    s32, s64 = v32.sum(axis=0)[ok], v64.sum(axis=0)[ok]
    np.testing.assert_allclose(s32, s64, rtol=0.02, atol=0.5)
