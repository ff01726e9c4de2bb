"""The header-only ParametricEngine drop-in (include/ucb_parametric_engine.hpp) compiles
against the reference's call pattern, links to libucb.so and reports errors the
reference's way (ok=false + message, no exception)."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import ucb
from helpers import LORENZ, ROSSLER, rk4_body

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    ucb.load()
    out = tmp_path_factory.mktemp("shim") / "shim_driver"
    subprocess.run(["g++", "-std=c++17", "-O1", f"-I{ROOT / 'include'}", str(ROOT / "tests" / "shim_driver.cpp"),
                    "-o", str(out), f"-L{ucb.HERE}", "-lucb", f"-Wl,-rpath,{ucb.HERE}"], check=True)
    return out


def run(driver, mode, body):
    return subprocess.run([str(driver), mode], input=body.encode(), capture_output=True, check=True).stdout.decode()


def test_shim_reports_validation_error(driver):
    out = run(driver, "invalid", rk4_body(ROSSLER))
    assert out.startswith("ok=0 error=n_pts must be > 0")


def test_shim_dft_and_fastsync_are_declared_and_not_supported(driver):
    # the session layer calls run_dft_1d / run_fastsync (analysis_session.cpp); the shim
    # declares them with the reference's types and answers ok=false with a message
    assert run(driver, "dft", rk4_body(LORENZ)).startswith("ok=0 error=run_dft_1d is not supported")
    assert run(driver, "fastsync", rk4_body(LORENZ)).startswith("ok=0 mode=1 error=run_fastsync is not supported")


@pytest.mark.gpu
def test_shim_cancel_token_stops_a_running_map(driver):
    # 1024^2 Rossler map with t_max = 2000 (about 1.1 s in FP64); the session's cancel token
    # is raised 150 ms in and the call must come back cancelled well before the map's time
    out = run(driver, "cancel", rk4_body(ROSSLER))
    kv = dict(p.split("=", 1) for p in out.split(" ")[:4])
    assert kv["ok"] == "0" and kv["cancelled"] == "1", out
    assert float(kv["ms"]) < 700, out
    assert 0.0 < float(kv["progress_at_cancel"]) < 1.0, out


def test_shim_rejects_continuation(driver):
    out = run(driver, "continuation", rk4_body(LORENZ))
    assert out.startswith("ok=0 error=continuation sweeps are not supported")


@pytest.mark.gpu
def test_shim_lle1d_equals_c_abi(driver):
    """run_lle_1d through the shim returns what ucb_run_lle1d returns."""
    out = run(driver, "lle1d", rk4_body(LORENZ)).splitlines()
    assert out[0].startswith("ok=1 error= n=16 lo=20 hi=200 idx=2") and "progress=1.0" in out[0]
    rows = [l.split() for l in out[1:]]
    eng = ucb.Engine(0)
    req = eng.lle1d_request(rk4_body(LORENZ), 3, (0.1, 0.1, 0.1), (0, 10.0, 28.0, 8.0 / 3.0), n_pts=16, param_index=2,
                            param_lo=20, param_hi=200, h=0.01, transient_time=5, t_max=20, NT=0.5,
                            opt=ucb.options(precision=ucb.PREC_F64))
    ref, flags = eng.run_lle1d(req)[:2]
    np.testing.assert_array_equal([float(r[0]) for r in rows], ref)
    np.testing.assert_array_equal([int(r[1]) for r in rows], flags)


@pytest.mark.gpu
def test_shim_ls1d_equals_c_abi(driver):
    """run_ls_1d through the shim returns ucb_run_ls1d's point-major spectrum as spectrum[i][k]."""
    out = run(driver, "ls1d", rk4_body(LORENZ)).splitlines()
    assert out[0].startswith("ok=1 error= n=10 k=3 idx=0")
    vals = np.array([float(l) for l in out[1:]])
    eng = ucb.Engine(0)
    req = eng.lle1d_request(rk4_body(LORENZ), 3, (0.1, 0.1, 0.1), (0, 10.0, 28.0, 8.0 / 3.0), n_pts=10,
                            sweep_over_var=True, var_sweep_index=0, param_lo=-5, param_hi=5, h=0.01,
                            transient_time=5, t_max=20, NT=0.5, opt=ucb.options(precision=ucb.PREC_F64))
    ref = eng.run_ls1d(req)[0]
    np.testing.assert_array_equal(vals, np.asarray(ref).ravel())


@pytest.mark.gpu
def test_shim_lle2d_runs(driver):
    out = run(driver, "lle2d", rk4_body(ROSSLER)).splitlines()
    assert out[0].startswith("ok=1 error= n=8")
    assert "progress=1.0" in out[0]
    vals = np.array([float(l.split()[0]) for l in out[1:]])
    assert len(vals) == 64 and np.isfinite(vals).all()


@pytest.mark.gpu
def test_shim_bif1d_runs(driver):
    out = run(driver, "bif1d", rk4_body(LORENZ)).splitlines()
    assert out[0].startswith("ok=1")
    counts = [int(l.split()[0]) for l in out[1:]]
    assert len(counts) == 8 and max(counts) > 0


@pytest.mark.gpu
def test_shim_ls2d_equals_c_abi(driver):
    """run_ls_2d through the shim returns what ucb_run_ls2d returns (plane-major spectrum)."""
    out = run(driver, "ls2d", rk4_body(LORENZ)).splitlines()
    assert out[0].startswith("ok=1 error= n=6 k=3")
    vals = np.array([float(l) for l in out[1:]])
    eng = ucb.Engine(0)
    req = eng.ls2d_request(rk4_body(LORENZ), 3, (0.1, 0.1, 0.1), (0, 10.0, 28.0, 8.0 / 3.0), n_pts=6, param_index=2,
                           param_index_2=1, param_lo=20, param_hi=40, param_lo_2=8.0, param_hi_2=12.0, h=0.01,
                           transient_time=5, t_max=20, NT=0.5, opt=ucb.options(precision=ucb.PREC_F64))
    ref, _, _ = eng.run_ls2d(req)
    np.testing.assert_array_equal(vals, ref.ravel())


@pytest.mark.gpu
def test_shim_bif2d_equals_c_abi(driver):
    """run_bifurcation_2d through the shim returns what ucb_run_bif2d returns."""
    out = run(driver, "bif2d", rk4_body(LORENZ)).splitlines()
    assert out[0].startswith("ok=1 error= n=6")
    vals = np.array([float(l.split()[0]) for l in out[1:]])
    eng = ucb.Engine(0)
    req = eng.bif2d_request(rk4_body(LORENZ), 3, (0.1, 0.1, 0.1), (0, 10.0, 28.0, 8.0 / 3.0), n_pts=6, param_index=2,
                            param_index_2=1, param_lo=20, param_hi=200, param_lo_2=5.0, param_hi_2=15.0, h=0.01,
                            transient_time=20, t_max=60, eps_dbscan=0.1)
    ref, _, _ = eng.run_bif2d(req)
    np.testing.assert_array_equal(vals, ref)


@pytest.mark.gpu
def test_shim_basins_equals_c_abi(driver):
    """run_basins / run_basins_recluster through the shim return what ucb_run_basins_dbscan
    returns (basin_idx, features, classes), and reclustering the cached features gives the
    same labels."""
    out = run(driver, "basins", rk4_body(LORENZ)).splitlines()
    assert out[0].startswith("ok=1 error= n=8") and "phase=2" in out[0]
    assert out[-1] == "recluster ok=1 same=1"
    rows = [l.split() for l in out[1:-1]]
    eng = ucb.Engine(0)
    req = eng.basins_dbscan_request(rk4_body(LORENZ), 3, (0.0, 0.0, 25.0), (0, 10.0, 10.0, 8.0 / 3.0), n_pts=8,
                                    axis_x_lo=-20, axis_x_hi=20, axis_y_lo=-20, axis_y_hi=20, h=0.01,
                                    transient_time=100, t_max=20, eps_dbscan=0.5)
    lab, f1, f2, cls, _ = eng.run_basins_dbscan(req)
    np.testing.assert_array_equal([int(r[0]) for r in rows], lab)
    np.testing.assert_array_equal([float(r[1]) for r in rows], f1)
    np.testing.assert_array_equal([float(r[2]) for r in rows], f2)
    np.testing.assert_array_equal([int(r[3]) for r in rows], cls)
