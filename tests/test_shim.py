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
