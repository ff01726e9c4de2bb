"""GPU parity of the LLE-2D path against the oracle (CPU restatement of LLEKernelCUDA +
run_lle_2d), through the C ABI.

Tolerances:
  * exact form (KRS body verbatim, no FMA contraction): trajectories bit-identical to the
    oracle; the only difference is the device vs glibc `log` (<= 1 ulp per block), so
    values agree to 1e-12 relative (FP64) / 1e-5 relative (FP32), flags exactly;
  * native FP64 (FMA-ordered RK4): trajectories within 1e-12 relative of the oracle
    before one Lyapunov time; on non-chaotic cells (oracle lambda < 0.01) |dLLE| <= 2e-3;
    on chaotic cells the difference is bounded by the intrinsic finite-time spread;
  * FP32 tangent form: same criteria as native FP64 on non-chaotic cells.
"""
import numpy as np
import pytest

import ucb
from helpers import LORENZ, engine_request, kernel_grid, lle2d_case, rk4_body
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    e = ucb.Engine(0)
    yield e
    e.close()


def oracle_lle(c, numb="f64"):
    return O.lle2d(O.Krs(c["body"], c["nx"], numb), kernel_grid(c))


def run(eng, c, **opt):
    v, f, res = eng.run_lle2d(engine_request(ucb, c, **opt))
    return v, f, res


def test_exact_f64_matches_oracle(eng):
    c = lle2d_case(n=16, t_max=20.0, transient=10.0)
    v, f, res = run(eng, c, precision=ucb.PREC_F64, mode=ucb.MODE_EXACT)
    ov, of = oracle_lle(c)
    np.testing.assert_array_equal(f, of)
    np.testing.assert_allclose(v, ov, rtol=1e-12, atol=1e-14)
    assert res.steps > 0 and res.kernel_ms > 0


def test_exact_f32_matches_oracle(eng):
    c = lle2d_case(n=12, t_max=10.0, transient=5.0)
    v, f, _ = run(eng, c, precision=ucb.PREC_F32, mode=ucb.MODE_EXACT)
    ov, of = oracle_lle(c, "f32")
    np.testing.assert_array_equal(f, of)
    np.testing.assert_allclose(v, ov, rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize("variant", ["pov0", "pov2", "pov2_swap", "log", "h_axis", "divergent"])
def test_exact_mapping_variants(eng, variant):
    base = lle2d_case(n=9, t_max=5.0, transient=2.0)
    if variant == "pov0":
        c = dict(base, sweep_over_var=True, sweep_over_var_2=True, var_sweep_index=0, var_sweep_index_2=2,
                 param_lo=-2.0, param_hi=2.0, param_lo_2=0.0, param_hi_2=3.0)
    elif variant == "pov2":
        c = dict(base, sweep_over_var=True, var_sweep_index=1, param_lo=-1.0, param_hi=1.0)
    elif variant == "pov2_swap":
        c = dict(base, sweep_over_var_2=True, var_sweep_index_2=1, param_index=3, param_lo=3.0, param_hi=9.0,
                 param_lo_2=-1.0, param_hi_2=1.0)
    elif variant == "log":
        c = dict(base, log_scale=True, log_scale_2=True, param_lo=0.05, param_hi=2.0)
    elif variant == "h_axis":
        c = dict(base, sweep_over_h=True, param_lo=0.005, param_hi=0.02)
    else:  # sweeping Rossler's a over [0.1, 1.5] sends part of the grid past max_value
        c = dict(base, param_index=1, param_lo=0.1, param_hi=1.5, max_value=50.0)
    v, f, _ = run(eng, c, precision=ucb.PREC_F64, mode=ucb.MODE_EXACT)
    ov, of = oracle_lle(c)
    np.testing.assert_array_equal(f, of)
    np.testing.assert_allclose(v, ov, rtol=1e-12, atol=1e-14)
    if variant == "divergent":
        assert (f == -1).any()


def test_native_f64_trajectory_parity_before_one_lyapunov_time(eng):
    # Rossler's largest exponent is <= ~0.2 on this grid: one Lyapunov time >= 5 time units.
    c = lle2d_case(n=8)
    req = engine_request(ucb, c, precision=ucb.PREC_F64, mode=ucb.MODE_NATIVE)
    n_steps = 400  # t = 4
    xs = eng.lle2d_states(req, n_steps)
    g = kernel_grid(c)
    k = O.Krs(c["body"], 3)
    ax0 = O.axis_values(c["n_pts"], c["param_lo"], c["param_hi"])
    ax1 = O.axis_values(c["n_pts"], c["param_lo_2"], c["param_hi_2"])
    for cell in range(c["n_pts"] ** 2):
        a = np.array(c["values"], dtype=np.float64)
        a[g["idx"][0]] = ax0[cell % c["n_pts"]]
        a[g["idx"][1]] = ax1[cell // c["n_pts"]]
        ref = k.steps(c["ic"], a, c["h"], n_steps)
        np.testing.assert_allclose(xs[cell], ref, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("prec,rtol", [(ucb.PREC_F64, 1e-11), (ucb.PREC_F32, 2e-4)])
def test_native_forced_system_trajectory_parity(eng, prec, rtol):
    """Forced Duffing (phase s with ds/dt = 1, 0.3 cos(s) in the right-hand side): the native
    step evaluates the forcing once per step (sincos) and rotates it to the stage phases; the
    states after 300 steps (t = 9.4, before the transient's sensitivity grows) agree with the
    oracle's RK4 of the verbatim body."""
    import math
    from helpers import DUFFING
    c = dict(body=rk4_body(DUFFING), nx=3, ic=(0.0, 0.0, 0.0), values=(0.0,), n_pts=6, sweep_over_var=True,
             sweep_over_var_2=True, var_sweep_index=0, var_sweep_index_2=1, param_index=1, param_index_2=1,
             param_lo=-1.5, param_hi=1.5, param_lo_2=-1.0, param_hi_2=1.0, h=2 * math.pi / 200,
             transient_time=1.0, t_max=2.0, NT=0.1, eps=1e-4, max_value=1e6)
    req = engine_request(ucb, c, precision=prec, mode=ucb.MODE_NATIVE)
    n_steps = 300
    xs = eng.lle2d_states(req, n_steps)
    k = O.Krs(c["body"], 3)
    ax0 = O.axis_values(6, -1.5, 1.5)
    ax1 = O.axis_values(6, -1.0, 1.0)
    for cell in range(36):
        x0 = np.array([ax0[cell % 6], ax1[cell // 6], 0.0])
        ref = k.steps(x0, np.array([0.0]), c["h"], n_steps)
        np.testing.assert_allclose(xs[cell], ref, rtol=rtol, atol=rtol)


def test_fp32_forced_clock_is_compensated(eng):
    """FP32 native form over a long horizon: the forced, damped linear oscillator
    x'' + 0.5 x' + x = cos(s), s' = 1 settles on x = 2 sin(t), v = 2 cos(t). After 3.5e5 steps
    (t ~ 1.1e4) a plain FP32 clock would have fallen ~30 rad behind (each add rounds to the
    ulp of the growing phase); the compensated clock stays within two ulps of n h, and the
    state within a few 1e-3 of FP64 (which is within 1e-4 of the closed form)."""
    import math
    body = ucb.codegen(r"\dot{x} = v \\ \dot{v} = -0.5 v - x + \cos(s) \\ \dot{s} = 1", "x,v,s")[0]
    h = 2 * math.pi / 200
    c = dict(body=body, nx=3, ic=(0.0, 0.0, 0.0), values=(0.0,), n_pts=4, sweep_over_var=True,
             sweep_over_var_2=True, var_sweep_index=0, var_sweep_index_2=1, param_index=1, param_index_2=1,
             param_lo=-1.0, param_hi=1.0, param_lo_2=-1.0, param_hi_2=1.0, h=h, transient_time=1.0, t_max=2.0,
             NT=0.1, eps=1e-4, max_value=1e6)
    n_steps = 350_000
    x32 = eng.lle2d_states(engine_request(ucb, c, precision=ucb.PREC_F32, mode=ucb.MODE_NATIVE), n_steps)
    x64 = eng.lle2d_states(engine_request(ucb, c, precision=ucb.PREC_F64, mode=ucb.MODE_NATIVE), n_steps)
    clock = n_steps * float(np.float32(h))
    ulp = float(np.spacing(np.float32(clock)))
    np.testing.assert_allclose(x32[:, 2], clock, atol=2 * ulp, rtol=0)
    t = n_steps * h
    np.testing.assert_allclose(x64[:, 0], 2 * math.sin(t), atol=1e-4)
    np.testing.assert_allclose(x64[:, 1], 2 * math.cos(t), atol=1e-4)
    np.testing.assert_allclose(x32[:, :2], x64[:, :2], atol=5e-3, rtol=0)


def test_exact_trajectory_bitwise(eng):
    c = lle2d_case(n=4)
    xs = eng.lle2d_states(engine_request(ucb, c, precision=ucb.PREC_F64, mode=ucb.MODE_EXACT), 3000)
    g = kernel_grid(c)
    k = O.Krs(c["body"], 3)
    ax0 = O.axis_values(4, c["param_lo"], c["param_hi"])
    ax1 = O.axis_values(4, c["param_lo_2"], c["param_hi_2"])
    for cell in range(16):
        a = np.array(c["values"], dtype=np.float64)
        a[g["idx"][0]] = ax0[cell % 4]
        a[g["idx"][1]] = ax1[cell // 4]
        np.testing.assert_array_equal(xs[cell], k.steps(c["ic"], a, c["h"], 3000))


@pytest.mark.parametrize("prec", [ucb.PREC_F64, ucb.PREC_F32])
def test_native_lle_within_tolerance(eng, prec):
    # Well-conditioned cells — those whose FP64 oracle exponent moves by < 1e-5 under a
    # 1e-7 relative perturbation of the swept parameters (the size of FP32 rounding):
    # fixed points, limit cycles, and chaotic cells not yet decorrelated at this horizon —
    # must agree with the FP64 oracle to 2e-3 on >= 99.5% of them. On the other cells no
    # arithmetic that is not bit-identical can: rounding differences are amplified until
    # the finite-time exponent is just another sample of the attractor. There the
    # engine's median difference must stay within 3x the oracle's own median change under
    # that perturbation.
    c = lle2d_case(n=24, t_max=200.0, transient=50.0)
    v, f, _ = run(eng, c, precision=prec, mode=ucb.MODE_NATIVE)
    ov, of = oracle_lle(c)
    np.testing.assert_array_equal(f, of)
    pert = dict(c, param_lo=c["param_lo"] * (1 + 1e-7), param_hi=c["param_hi"] * (1 + 1e-7),
                param_lo_2=c["param_lo_2"] * (1 + 1e-7), param_hi_2=c["param_hi_2"] * (1 + 1e-7))
    pv, _ = oracle_lle(pert)
    d = np.abs(v - ov)
    spread = np.abs(pv - ov)
    quiet = spread < 1e-5
    assert quiet.sum() > 20 and (~quiet).sum() > 20
    assert np.mean(d[quiet] <= 2e-3) >= 0.995, np.sort(d[quiet])[-5:]
    assert np.median(d[~quiet]) <= 3 * np.median(spread[~quiet]) + 1e-3


def test_lorenz_grid_native_runs(eng):
    c = dict(lle2d_case(n=8, t_max=20.0, transient=5.0), body=rk4_body(LORENZ), values=(0, 10.0, 28.0, 8 / 3),
             param_index=1, param_index_2=2, param_lo=5.0, param_hi=15.0, param_lo_2=20.0, param_hi_2=40.0,
             ic=(0.1, 0.1, 0.1))
    v, f, _ = run(eng, c, precision=ucb.PREC_F64, mode=ucb.MODE_NATIVE)
    ov, of = oracle_lle(c)
    np.testing.assert_array_equal(f, of)
    assert np.isfinite(v).all()


def test_device_entry_matches_host_entry(eng):
    torch = pytest.importorskip("torch")
    c = lle2d_case(n=10, t_max=5.0, transient=2.0)
    req = engine_request(ucb, c, precision=ucb.PREC_F64, mode=ucb.MODE_EXACT)
    hv, hf, _ = eng.run_lle2d(req)
    dv = torch.empty(100, dtype=torch.float64, device="cuda")
    df = torch.empty(100, dtype=torch.int32, device="cuda")
    s = torch.cuda.current_stream()
    eng.lle2d_device(req, dv.data_ptr(), df.data_ptr(), s.cuda_stream)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(dv.cpu().numpy(), hv)
    np.testing.assert_array_equal(df.cpu().numpy(), hf)


@pytest.mark.parametrize("n", [33, 48])
def test_fp32_paired_cells_match_one_cell_per_thread(eng, n):
    """paired_cells: the FP32 tangent kernel integrates two cells per thread in packed FP32
    pairs (FFMA2 / FADD2 / FMUL2), the same arithmetic as one cell per thread with scalar
    instructions: flags and exponents bit-identical (33^2 leaves an odd tail pair with one
    cell), the same step count."""
    c = lle2d_case(n=n, t_max=20.0, transient=10.0)
    v2, f2, r2 = eng.run_lle2d(engine_request(ucb, c, precision=ucb.PREC_F32, paired_cells=True))
    v1, f1, r1 = eng.run_lle2d(engine_request(ucb, c, precision=ucb.PREC_F32))
    np.testing.assert_array_equal(f2, f1)
    np.testing.assert_array_equal(v2, v1)
    assert r2.steps == r1.steps
