"""LLE 1D / LS 1D (run_lle_1d / run_ls_1d): the LLE and spectrum kernels over one swept
axis. A 1-D sweep is the first row of a 2-D map whose second axis is pinned to the base
value (same cell index, hence the same probe subsequence), so the oracle's 2-D
restatement over cells 0..n-1 is the reference; the exact form matches it to 1e-12."""
import numpy as np
import pytest

import ucb
from helpers import LORENZ, ROSSLER, kernel_grid, lle2d_case, rk4_body
from oracle import oracle as O


def line_case(**kw):
    c = lle2d_case(n=24, t_max=20.0, transient=5.0)
    c.update(param_index_2=3, param_lo_2=5.7, param_hi_2=5.7)   # second axis pinned to c = 5.7
    c.update(kw)
    return c


def request(c, **opt):
    return ucb.Engine.lle1d_request(c["body"], c["nx"], c["ic"], c["values"], n_pts=c["n_pts"],
                                    param_index=c["param_index"], param_lo=c["param_lo"], param_hi=c["param_hi"],
                                    sweep_over_var=c.get("sweep_over_var", False),
                                    var_sweep_index=c.get("var_sweep_index", 0),
                                    log_scale=c.get("log_scale", False), h=c["h"], transient_time=c["transient_time"],
                                    t_max=c["t_max"], NT=c["NT"], eps=c["eps"], max_value=c["max_value"],
                                    csv_output_path=c.get("csv"), opt=ucb.options(**opt))


def test_lle1d_validation_messages():
    eng = ucb.Engine(0)
    c = line_case()
    for field, value, msg in (("n_pts", 0, "n_pts must be > 0"), ("param_index", 9, "param_index out of range"),
                              ("NT", 0.0, "NT must be > 0")):
        r = request(c)
        setattr(r, field, value)
        with pytest.raises(ucb.UcbError, match=msg):
            eng.run_lle1d(r)
    eng.close()


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["param", "log", "ic"])
def test_lle1d_exact_matches_oracle_row(variant, tmp_path):
    eng = ucb.Engine(0)
    kw = {}
    if variant == "log":
        kw = dict(log_scale=True, param_lo=0.1, param_hi=1.5)
    elif variant == "ic":
        kw = dict(sweep_over_var=True, var_sweep_index=0, param_lo=-2.0, param_hi=2.0)
    c = line_case(csv=str(tmp_path / "lle1d.csv"), **kw)
    v, f, res = eng.run_lle1d(request(c, precision=ucb.PREC_F64, mode=ucb.MODE_EXACT))
    g = dict(c)
    if variant == "ic":   # mixed 2-D map: axis 0 an initial condition, axis 1 the pinned parameter
        g.update(sweep_over_var=True, sweep_over_var_2=False)
    ov, of = O.lle2d(O.Krs(c["body"], 3), kernel_grid(g), cells=np.arange(c["n_pts"]))
    np.testing.assert_array_equal(f, of)
    ok = of == 1
    np.testing.assert_allclose(v[ok], ov[ok], rtol=1e-12, atol=1e-14)
    assert np.isnan(v[~ok]).all()
    rows = (tmp_path / "lle1d.csv").read_text().strip().splitlines()
    assert len(rows) == c["n_pts"] and rows[0].count(",") == 1
    assert (tmp_path / "lle1d.csv_config.csv").read_text().startswith("1D LLE\nParameter estimation\n")
    eng.close()


@pytest.mark.gpu
def test_ls1d_exact_matches_oracle_row():
    eng = ucb.Engine(0)
    c = line_case(body=rk4_body(LORENZ), ic=(0.1, 0.1, 0.1), values=(0, 10.0, 28.0, 8 / 3), param_index=2,
                  param_lo=20.0, param_hi=40.0, param_index_2=1, param_lo_2=10.0, param_hi_2=10.0, NT=0.5,
                  eps=1e-6)
    vals, flags, res = eng.run_ls1d(request(c, precision=ucb.PREC_F64, mode=ucb.MODE_EXACT))
    ov, of = O.ls2d(O.Krs(c["body"], 3), kernel_grid(c), cells=np.arange(c["n_pts"]))
    ov = ov.reshape(c["n_pts"], 3)
    np.testing.assert_array_equal(flags, of)
    np.testing.assert_allclose(vals, ov, rtol=1e-12, atol=1e-12)
    assert res.n_exponents == 3
    # Lorenz divergence: the spectrum sums to -(sigma + 1 + beta) times the reference's step
    # factor (NT/h + 1) / (NT/h) = 51/50 (one extra step per block)
    s = vals[flags == 1].sum(axis=1)
    assert np.all(np.abs(s + 51 / 50 * (10 + 1 + 8 / 3)) < 0.05)
    eng.close()
