"""CPU tests of the oracle: pins against the reference's own material (no GPU)."""
import numpy as np
import pytest

from helpers import LORENZ, ROSSLER, codegen_cases, kernel_grid, lle2d_case, rk4_body
from oracle import oracle as O


def test_rng_stub_constants():
    # lle2d.template.cu:45-56 == parametric_engine.cpp:196-209: splitmix64 init, LCG uniform.
    mask = (1 << 64) - 1

    def ref(seq, n):
        z = (1234567891 + seq * 0x9E3779B97F4A7C15) & mask
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & mask
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & mask
        s = z ^ (z >> 31)
        out = []
        for _ in range(n):
            s = (s * 6364136223846793005 + 1442695040888963407) & mask
            out.append(np.float32(((s >> 40) & 0xFFFFFF) + 1) / np.float32(16777216.0))
        return np.array(out, dtype=np.float32)

    for seq in (0, 1, 7, 123456, 1048575):
        np.testing.assert_array_equal(O.rng_uniforms(seq, 8), ref(seq, 8))


def test_axis_values_formula():
    # getValueByIdx (cudaLibrary.cu:1344-1361): (1 - t) lo + t hi, t = i / (n - 1)
    v = O.axis_values(5, 2.0, 20.0)
    t = np.arange(5) / 4.0
    np.testing.assert_array_equal(v, (1 - t) * 2.0 + t * 20.0)
    assert O.axis_values(1, 3.0, 7.0)[0] == 7.0  # nPts == 1 returns the upper end


def test_rossler_golden_body_steps_like_hand_written_model():
    # cudaLibrary.cu:129-159 is a hand-written Rossler RK4 with a[1..3] = a, b, c; the
    # codegen body for the Rossler preset must integrate identically.
    body = rk4_body("library_Rossler")
    k = O.Krs(body, 3)
    x = k.steps([1.0, 1.0, 1.0], [0, 0.2, 0.2, 5.7], 0.01, 1000)

    def rhs(X, a):
        return np.array([-X[1] - X[2], X[0] + a[1] * X[1], a[2] + X[2] * (X[0] - a[3])])

    X = np.array([1.0, 1.0, 1.0])
    a = [0, 0.2, 0.2, 5.7]
    h = 0.01
    for _ in range(1000):
        X1 = X.copy()
        kk = []
        for j in range(4):
            kj = rhs(X1, a)
            kk.append(kj)
            if j == 3:
                X = X + h * (kk[0] + 2 * kk[1] + 2 * kk[2] + kk[3]) / 6
            elif j == 2:
                X1 = X + h * kj
            else:
                X1 = X + 0.5 * h * kj
    np.testing.assert_array_equal(x, X)


def test_rossler_lle_known_value():
    # Textbook largest exponent of Rossler (a=b=0.2, c=5.7) is about 0.071. The reference
    # semantics advance every NT block by NT/h + 1 steps but divide by t_max, so the
    # estimate carries the factor (NT/h + 1)/(NT/h) = 1.1.
    c = lle2d_case(n=1, t_max=1000.0, transient=100.0, param_lo=0.2, param_hi=0.2, param_lo_2=5.7, param_hi_2=5.7)
    v, f = O.lle2d(O.Krs(c["body"], 3), kernel_grid(c))
    assert f[0] == 1
    assert abs(v[0] / 1.1 - 0.0714) < 0.005


def test_lorenz_lle_known_value():
    c = dict(lle2d_case(n=1, t_max=500.0, transient=50.0), body=rk4_body(LORENZ), values=(0, 10.0, 28.0, 8.0 / 3.0),
             param_index=1, param_index_2=2, param_lo=10.0, param_hi=10.0, param_lo_2=28.0, param_hi_2=28.0,
             ic=(0.1, 0.1, 0.1))
    v, f = O.lle2d(O.Krs(c["body"], 3), kernel_grid(c))
    assert abs(v[0] / 1.1 - 0.906) < 0.05


def test_lorenz_spectrum_sum():
    # Sum of the Lyapunov spectrum equals the divergence -(sigma + 1 + beta) = -13.667.
    c = dict(lle2d_case(n=1, t_max=200.0, transient=20.0, NT=0.1), body=rk4_body(LORENZ),
             values=(0, 10.0, 28.0, 8.0 / 3.0), param_index=1, param_index_2=2, param_lo=10.0, param_hi=10.0,
             param_lo_2=28.0, param_hi_2=28.0, ic=(0.1, 0.1, 0.1), eps=1e-6)
    v, f = O.ls2d(O.Krs(c["body"], 3), kernel_grid(c))
    assert f[0] == 1
    assert abs(v.sum() / 1.1 - (-(10 + 1 + 8 / 3))) < 0.2


def test_divergent_cell_flags():
    # A parameter that blows up the trajectory ends with the 999 sentinel and flag -1.
    c = lle2d_case(n=2, t_max=5.0, param_lo=0.05, param_hi=0.05, param_lo_2=2.0, param_hi_2=2.0,
                   values=(0, 5.0, 0.2, 5.7), param_index=2, param_index_2=3, max_value=1e3)
    v, f = O.lle2d(O.Krs(c["body"], 3), kernel_grid(c))
    assert (v == 999.0).all() and (f == -1).all()


def test_float_and_double_numb_agree_short_horizon():
    body = rk4_body(ROSSLER)
    x64 = O.Krs(body, 3, "f64").steps([1, 1, 1], [0, 0.2, 0.2, 5.7], 0.01, 200)
    x32 = O.Krs(body, 3, "f32").steps([1, 1, 1], [0, 0.2, 0.2, 5.7], 0.01, 200)
    np.testing.assert_allclose(x32, x64, rtol=1e-4)


def test_peak_finder_streaming_semantics_on_known_series():
    # Bifurcation of Lorenz at rho=28 (chaotic) and rho=160 (period-2 window): peaks > 0.
    body = rk4_body(LORENZ)
    b = dict(n_pts=2, sweep_index=2, lo=28.0, hi=160.0, ic=(0.1, 0.1, 0.1), values=(0, 10.0, 28.0, 8 / 3),
             h=0.01, transient_time=20.0, t_max=50.0, max_value=1e6)
    counts, peaks, intervals = O.bif1d(O.Krs(body, 3), b, max_out=64)
    assert (counts > 5).all()
    assert np.isfinite(peaks[0, :min(counts[0], 64)]).all()
    assert (intervals[0, :min(counts[0], 64)] > 0).all()
