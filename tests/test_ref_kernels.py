"""Parity pinned to the reference's own kernels, run on the GPU.

oracle/build_ref_kernels.py compiles the reference's NVRTC templates (lle2d, ls2d,
bifurcation1d + cudaLibrary.cu) unchanged, with the reference's compile options, and
oracle/ref_harness.cpp launches them with the reference driver's host logic. Two builds:

  * "nofma": the reference's options plus --fmad=false. Every operation rounds once, as in
    the engine's exact form (KRS body verbatim, compiled without contraction) and in the
    oracle (g++ -ffp-contract=off), and the device type is the reference's own
    `numb = float`. The engine's exact FP32 form must equal the reference kernel BIT FOR
    BIT (values and flags: both take the same device `log` of the same float); the oracle
    at numb=float must agree to 1e-5 relative (its glibc `logf` may differ from the
    device's by one ulp per block; the trajectories are the same).
  * "stock": the reference's options exactly as it ships them (FMA contraction on). Its
    trajectories part from the contraction-free ones at the rounding level, so it is
    compared with tolerances stated per test.

Skipped only when the reference modules were not built (the build needs the reference
tree; oracle/build_ref.sh).
"""
import numpy as np
import pytest

import ucb
from helpers import HYPER_ROSSLER, LORENZ, engine_request, kernel_grid, lle2d_case, rk4_body
from oracle import oracle as O
from oracle import ref_kernels as R

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not R.available(), reason="reference kernels not built (oracle/build_ref.sh)")]


@pytest.fixture(scope="module")
def eng():
    e = ucb.Engine(0)
    yield e
    e.close()


def lle_cases():
    base = lle2d_case(n=16, t_max=20.0, transient=10.0)
    lorenz = lle2d_case(n=12, t_max=10.0, transient=5.0, body=rk4_body(LORENZ), ic=(0.1, 0.1, 0.1),
                        values=(0, 10.0, 28.0, 8 / 3), sweep_over_var=True, sweep_over_var_2=True,
                        var_sweep_index=0, var_sweep_index_2=2, param_lo=-10.0, param_hi=10.0, param_lo_2=5.0,
                        param_hi_2=40.0, eps=1e-3)
    pov2 = lle2d_case(n=12, t_max=10.0, transient=5.0, sweep_over_var=True, var_sweep_index=0, param_lo=-3.0,
                      param_hi=3.0)
    return {"lle2d_rossler_pov1": base, "lle2d_lorenz_pov0": lorenz, "lle2d_rossler_pov2": pov2}


@pytest.mark.parametrize("case", list(lle_cases()))
def test_lle_engine_exact_f32_equals_reference_kernel(eng, case):
    c = lle_cases()[case]
    g = kernel_grid(c)
    assert not g["swap_xy"]
    rv, rf, _ = R.lle2d(case, "nofma", g)
    v, f, _ = eng.run_lle2d(engine_request(ucb, c, precision=ucb.PREC_F32, mode=ucb.MODE_EXACT))
    np.testing.assert_array_equal(f, rf)
    np.testing.assert_array_equal(v, rv)
    assert (rf == 1).sum() > 0


@pytest.mark.parametrize("case", list(lle_cases()))
def test_lle_oracle_f32_matches_reference_kernel(case):
    c = lle_cases()[case]
    g = kernel_grid(c)
    rv, rf, _ = R.lle2d(case, "nofma", g)
    ov, of = O.lle2d(O.Krs(c["body"], c["nx"], "f32"), g)
    np.testing.assert_array_equal(of, rf)
    np.testing.assert_allclose(ov, rv, rtol=1e-5, atol=1e-6)


def hyper_case(**kw):
    d = lle2d_case(n=6, body=rk4_body(HYPER_ROSSLER), nx=4, ic=(-10.0, -6.0, 0.0, 10.0), values=(0, 0.25, 0.05),
                   param_index=1, param_index_2=2, param_lo=0.1, param_hi=0.35, param_lo_2=0.01, param_hi_2=0.1,
                   h=0.01, transient_time=5.0, t_max=10.0, NT=0.1, eps=1e-3)
    d.update(kw)
    return d


def lorenz_ls_case(**kw):
    d = lle2d_case(n=4, body=rk4_body(LORENZ), nx=3, ic=(0.1, 0.1, 0.1), values=(0, 10.0, 28.0, 8 / 3),
                   param_index=1, param_index_2=2, param_lo=9.0, param_hi=11.0, param_lo_2=26.0, param_hi_2=30.0,
                   h=0.01, transient_time=5.0, t_max=20.0, NT=0.1, eps=1e-3)
    d.update(kw)
    return d


LS_CASES = {"ls2d_hyper_rossler_pov1": hyper_case, "ls2d_lorenz_pov1": lorenz_ls_case}


def ls_request(c, **opt):
    kw = {k: c[k] for k in ("n_pts", "param_index", "param_index_2", "param_lo", "param_hi", "param_lo_2",
                             "param_hi_2", "h", "transient_time", "t_max", "NT", "eps", "max_value")}
    return ucb.Engine.ls2d_request(c["body"], c["nx"], c["ic"], c["values"], method=ucb.LS_FIXED,
                                   opt=ucb.options(**opt), **kw)


@pytest.mark.parametrize("case", list(LS_CASES))
def test_ls_engine_exact_f32_equals_reference_kernel(eng, case):
    c = LS_CASES[case]()
    g = kernel_grid(c)
    rv, rf, _ = R.lle2d(case, "nofma", g, ls=True)
    v, f, _ = eng.run_ls2d(ls_request(c, precision=ucb.PREC_F32, mode=ucb.MODE_EXACT))
    np.testing.assert_array_equal(f, rf)
    np.testing.assert_array_equal(v, rv.T)
    ov, of = O.ls2d(O.Krs(c["body"], c["nx"], "f32"), g)
    np.testing.assert_array_equal(of, rf)
    np.testing.assert_allclose(ov.reshape(c["nx"], -1), rv.T, rtol=1e-5, atol=1e-5)


def bif_case(**kw):
    d = dict(n_pts=64, sweep_kind=0, sweep_index=2, lo=20.0, hi=200.0, log_scale=False, ic=(0.1, 0.1, 0.1),
             values=(0, 10.0, 28.0, 8 / 3), h=0.01, transient_time=10.0, t_max=40.0, pre_scaller=1,
             writable_var=0, max_value=1e6)
    d.update(kw)
    return d


def engine_bif(eng, b, body, cap=64, **opt):
    req = ucb.Engine.bif1d_request(body, 3, b["ic"], b["values"], n_pts=b["n_pts"],
                                   param_index=b["sweep_index"] if b["sweep_kind"] == 0 else 1,
                                   param_lo=b["lo"], param_hi=b["hi"], h=b["h"], transient_time=b["transient_time"],
                                   t_max=b["t_max"], writable_var=b["writable_var"], pre_scaller=b["pre_scaller"],
                                   max_value=b["max_value"], max_peaks=cap, sweep_over_var=b["sweep_kind"] == 1,
                                   var_sweep_index=b["sweep_index"] if b["sweep_kind"] == 1 else 0,
                                   log_scale=b["log_scale"], opt=ucb.options(**opt))
    counts, peaks, intervals, _ = eng.run_bif1d(req)
    return counts, peaks, intervals


BIF_CASES = {
    "lorenz_64": ("bif1d_lorenz_pov1", LORENZ, bif_case()),
    "lorenz_prescaller_combo": ("bif1d_lorenz_pov1", LORENZ, bif_case(pre_scaller=3, t_max=60.0, writable_var=-1)),
    # the bifurcation configuration at full size: 1024 values of rho in [20, 200],
    # 5,000 transient + 20,000 recorded steps
    "lorenz_full_1024": ("bif1d_lorenz_pov1", LORENZ, bif_case(n_pts=1024, transient_time=50.0, t_max=200.0)),
    "rossler_ic_sweep": ("bif1d_rossler_pov0", "rossler_config",
                         bif_case(sweep_kind=1, sweep_index=0, lo=-5.0, hi=5.0, ic=(1.0, 1.0, 1.0),
                                  values=(0, 0.2, 0.2, 5.7), t_max=100.0)),
}


@pytest.mark.parametrize("name", list(BIF_CASES))
def test_bif_engine_exact_f32_equals_reference_kernel(eng, name):
    case, system, b = BIF_CASES[name]
    body = rk4_body(system)
    rc, rp, ri, _ = R.bif1d(case, "nofma", b)
    counts, peaks, intervals = engine_bif(eng, b, body, precision=ucb.PREC_F32, mode=ucb.MODE_EXACT)
    np.testing.assert_array_equal(counts, rc)
    np.testing.assert_array_equal(np.isfinite(peaks), np.isfinite(rp))
    m = np.isfinite(rp)
    np.testing.assert_array_equal(peaks[m], rp[m])
    np.testing.assert_array_equal(intervals[m], ri[m])
    assert (rc > 0).any()


@pytest.mark.parametrize("name", ["lorenz_64", "rossler_ic_sweep"])
def test_bif_oracle_f32_equals_reference_kernel(name):
    case, system, b = BIF_CASES[name]
    rc, rp, ri, _ = R.bif1d(case, "nofma", b)
    oc, op, oi = O.bif1d(O.Krs(rk4_body(system), 3, "f32"), b, max_out=64)
    np.testing.assert_array_equal(oc, rc)
    m = np.isfinite(rp)
    np.testing.assert_array_equal(np.isfinite(op), m)
    np.testing.assert_array_equal(op[m], rp[m])
    np.testing.assert_array_equal(oi[m], ri[m])


def test_engine_beats_reference_kernel_on_the_headline_map(eng):
    """The headline map (Rossler 1024^2, 1e4 transient + 1e5 measured steps, renormalised
    every 10) through the reference's own LLE kernel as it ships (numb = float, FMA
    contraction on) and through the engine on the same GPU: the engine's FP32 form takes
    less than half the reference kernel's time and, against the exact FP64 map, keeps at
    least as many cells within 2e-3."""
    c = lle2d_case(n=1024, t_max=1000.0, transient=100.0)
    g = kernel_grid(c)
    rv, rf, ref_ms = R.lle2d("lle2d_rossler_pov1", "stock", g)
    eng.run_lle2d(engine_request(ucb, lle2d_case(n=8), precision=ucb.PREC_F32))  # compile outside the timing
    v32, f32, r32 = eng.run_lle2d(engine_request(ucb, c, precision=ucb.PREC_F32))
    v64, f64, _ = eng.run_lle2d(engine_request(ucb, c, precision=ucb.PREC_F64, mode=ucb.MODE_EXACT))
    ok = (f64 == 1) & (rf == 1) & (f32 == 1)

    def within(v):
        return float(np.mean(np.abs(v[ok] - v64[ok]) <= 2e-3))

    print(f"reference kernel (shipped build) {ref_ms:.1f} ms, engine FP32 {r32.kernel_ms:.1f} ms "
          f"({ref_ms / r32.kernel_ms:.2f}x); within 2e-3 of exact FP64: reference {within(rv):.4f}, "
          f"engine FP32 {within(v32):.4f} over {int(ok.sum())} cells")
    assert ok.sum() > 0.9 * ok.size
    assert r32.kernel_ms < 0.5 * ref_ms
    assert within(v32) >= within(rv)
