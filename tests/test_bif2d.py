"""Bifurcation 2D period maps (run_bif2d): per cell the trajectory and peaks of the 1-D
diagram, then the reference's dbscan of the peak values. The exact form records
bit-identical series, so peaks, dbscan clusters and periods equal the oracle's cell for
cell; the native forms agree on the share of cells."""
import numpy as np
import pytest

import ucb
from helpers import LORENZ, kernel_grid, rk4_body
from oracle import oracle as O


def case(**kw):
    d = dict(body=rk4_body(LORENZ), nx=3, ic=(0.1, 0.1, 0.1), values=(0, 10.0, 28.0, 8 / 3), n_pts=12,
             param_index=2, param_index_2=1, param_lo=20.0, param_hi=200.0, param_lo_2=5.0, param_hi_2=15.0,
             h=0.01, transient_time=20.0, t_max=60.0, NT=1.0, eps=1.0, max_value=1e6, pre_scaller=1,
             writable_var=0, eps_dbscan=0.1)
    d.update(kw)
    return d


def request(c, **opt):
    keys = ("n_pts", "param_index", "param_index_2", "var_sweep_index", "var_sweep_index_2", "sweep_over_var",
            "sweep_over_var_2", "sweep_over_h", "sweep_over_h_2", "log_scale", "log_scale_2", "param_lo", "param_hi",
            "param_lo_2", "param_hi_2", "writable_var", "h", "transient_time", "t_max", "pre_scaller", "max_value",
            "eps_dbscan")
    return ucb.Engine.bif2d_request(c["body"], c["nx"], c["ic"], c["values"], csv_output_path=c.get("csv"),
                                    opt=ucb.options(**opt), **{k: c[k] for k in keys if k in c})


def oracle(c, numb="f64"):
    return O.bif2d(O.Krs(c["body"], 3, numb), kernel_grid(c), c["eps_dbscan"], pre_scaller=c["pre_scaller"],
                   writable_var=c["writable_var"])


def test_bif2d_validation_messages():
    eng = ucb.Engine(0)
    for field, value, msg in (("eps_dbscan", 0.0, "eps_dbscan must be > 0"),
                              ("pre_scaller", 0, "pre_scaller must be > 0"),
                              ("writable_var", 3, "writable_var out of range"),
                              ("n_pts", 0, "n_pts must be > 0")):
        with pytest.raises(ucb.UcbError, match=msg):
            eng.run_bif2d(request(case(**{field: value})))
    with pytest.raises(ucb.UcbError, match="h lo/hi must be > 0"):
        eng.run_bif2d(request(case(sweep_over_h=True, param_lo=0.0, param_hi=0.02)))
    eng.close()


@pytest.mark.parametrize("rho,expected", [(20.0, -1), (250.0, 1), (28.0, None)])
def test_oracle_period_regimes(rho, expected):
    """Known Lorenz regimes through the restated dbscan: a stable fixed point keeps the
    trajectory's fixed-point flag (-1); a period-1 orbit (all peaks within eps) gives 1,
    because the reference's inner loop never visits the last peak, which then opens a
    second cluster, and the result is the cluster count minus one; the chaotic attractor
    gives many clusters."""
    c = case(n_pts=1, values=(0, 10.0, rho, 8 / 3), param_lo=rho, param_hi=rho, param_lo_2=10.0, param_hi_2=10.0,
             transient_time=200.0, t_max=100.0)
    v, f = oracle(c)
    if expected is None:
        assert f[0] == 1 and v[0] > 10
    else:
        assert v[0] == expected and f[0] == (1 if expected >= 0 else -1)


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["base", "mixed", "swap", "h_sweep", "log", "combo_prescaller"])
def test_bif2d_exact_matches_oracle(variant, tmp_path):
    eng = ucb.Engine(0)
    kw = {}
    if variant == "mixed":
        kw = dict(sweep_over_var=True, var_sweep_index=0, param_lo=-5.0, param_hi=5.0)
    elif variant == "swap":
        kw = dict(sweep_over_var_2=True, var_sweep_index_2=2, param_lo_2=1.0, param_hi_2=30.0)
    elif variant == "h_sweep":
        kw = dict(sweep_over_h=True, param_lo=0.005, param_hi=0.02)
    elif variant == "log":
        kw = dict(log_scale=True, log_scale_2=True, param_lo=20.0, param_hi=200.0)
    elif variant == "combo_prescaller":
        kw = dict(writable_var=-1, pre_scaller=2, eps_dbscan=0.5)
    c = case(csv=str(tmp_path / "bif2d.csv"), **kw)
    v, f, res = eng.run_bif2d(request(c, precision=ucb.PREC_F64, mode=ucb.MODE_EXACT))
    ov, of = oracle(c)
    np.testing.assert_array_equal(f, of)
    np.testing.assert_array_equal(v, ov)
    assert res.max_val == ov[(of == 1) & (ov >= 0)].max()
    grid = (tmp_path / "bif2d.csv").read_text().strip().splitlines()
    assert len(grid) == c["n_pts"] and grid[0].count(",") == c["n_pts"] - 1
    assert (tmp_path / "bif2d.csv_config.csv").read_text().startswith("2D bifurcation (DBSCAN)\n")
    eng.close()


@pytest.mark.gpu
def test_bif2d_exact_f32_matches_oracle():
    eng = ucb.Engine(0)
    c = case(n_pts=10)
    v, f, _ = eng.run_bif2d(request(c, precision=ucb.PREC_F32, mode=ucb.MODE_EXACT))
    ov, of = oracle(c, "f32")
    np.testing.assert_array_equal(f, of)
    np.testing.assert_array_equal(v, ov)
    eng.close()


@pytest.mark.gpu
def test_bif2d_native_forms_agree_on_regular_cells():
    eng = ucb.Engine(0)
    c = case(n_pts=16, t_max=100.0)
    ov, of = oracle(c)
    for prec in (ucb.PREC_F64, ucb.PREC_F32):
        v, f, _ = eng.run_bif2d(request(c, precision=prec, mode=ucb.MODE_NATIVE))
        # periodic / fixed-point cells (few clusters) keep their period; chaotic cells
        # (many clusters) stay chaotic
        regular = (of == 1) & (ov <= 4)
        assert (v[regular] == ov[regular]).mean() > 0.9
        assert ((v > 4) == (ov > 4)).mean() > 0.9
    eng.close()
