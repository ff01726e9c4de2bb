"""CSV wire format pinned to the reference's own writers, byte for byte.

oracle/_ref/ref_csv is the reference's data_export.cpp compiled as-is (oracle/build_ref.sh)
behind a driver that fills the snapshots the way the reference's run_* paths do. Each test
runs a map through the engine with csv_output_path set, hands the engine's own result
arrays to the reference's writers, and requires every file (the *_config.csv header and
the data files) to be identical. The engine runs in its FP32 form: the reference's numb is
float, so its config files print a[] and X0[] (and the 1-D ranges) narrowed to float, as the
engine does for its FP32 form.

Skipped only when the reference's writers were not built (the build needs the reference tree).
"""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import ucb
from helpers import HYPER_ROSSLER, LORENZ, ROSSLER, rk4_body

ROOT = Path(__file__).resolve().parents[1]
REF_CSV = ROOT / "oracle" / "_ref" / "ref_csv"

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not REF_CSV.exists(), reason="reference CSV writers not built")]

F32 = dict(precision=ucb.PREC_F32)


@pytest.fixture(scope="module")
def eng():
    e = ucb.Engine(0)
    yield e
    e.close()


def write_spec(d: Path, kind: str, **kv) -> Path:
    lines = [f"kind {kind}", f"path {d / 'ref.csv'}"]
    for k, v in kv.items():
        if isinstance(v, np.ndarray):
            f = d / f"{k}.bin"
            v.tofile(f)
            lines.append(f"{k} {f}")
        elif isinstance(v, (list, tuple)):
            lines.append(f"{k} " + " ".join(repr(float(x)) for x in v))
        else:
            lines.append(f"{k} {v!r}" if isinstance(v, float) else f"{k} {v}")
    p = d / "spec.txt"
    p.write_text("\n".join(lines) + "\n")
    return p


def assert_same_files(d: Path, suffixes):
    subprocess.run([str(REF_CSV), str(d / "spec.txt")], check=True)
    for suf in suffixes:
        ours = (d / ("eng.csv" + suf)).read_bytes()
        ref = (d / ("ref.csv" + suf)).read_bytes()
        assert ours == ref, f"{suf or 'data'} differs:\n{ours[:400]!r}\n{ref[:400]!r}"


ROSSLER_MAP = dict(ic=(1.0, 1.0, 1.0), values=(0.0, 0.2, 0.2, 5.7), param_index=2, param_index_2=3, param_lo=0.05,
                   param_hi=2.0, param_lo_2=2.0, param_hi_2=20.0, h=0.01, transient_time=5.0, t_max=10.0, NT=0.1,
                   eps=1e-4)


@pytest.mark.parametrize("variant", ["pov1", "pov0", "pov2"])
def test_lle2d_files_equal_reference_writer(eng, tmp_path, variant):
    kw = dict(ROSSLER_MAP)
    if variant == "pov0":
        kw.update(sweep_over_var=True, sweep_over_var_2=True, var_sweep_index=0, var_sweep_index_2=2,
                  param_lo=-2.0, param_hi=2.0, param_lo_2=-1.0, param_hi_2=1.5)
    elif variant == "pov2":
        kw.update(sweep_over_var=True, var_sweep_index=1, param_lo=-3.0, param_hi=3.0)
    req = ucb.Engine.lle2d_request(rk4_body(ROSSLER), 3, n_pts=9, csv_output_path=str(tmp_path / "eng.csv"),
                                   opt=ucb.options(**F32), **{k: v for k, v in kw.items() if k not in ("ic", "values")},
                                   initial_conditions=kw["ic"], base_values=kw["values"])
    v, f, _ = eng.run_lle2d(req)
    pov = {"pov1": 1, "pov0": 0, "pov2": 2}[variant]
    idx1 = kw.get("var_sweep_index", 0) if kw.get("sweep_over_var") else kw["param_index"]
    idx2 = kw.get("var_sweep_index_2", 0) if kw.get("sweep_over_var_2") else kw["param_index_2"]
    write_spec(tmp_path, "lle2d", n_pts=9, values=kw["values"], ic=kw["ic"], par_or_var=pov, tMax=kw["t_max"],
               NT=kw["NT"], transient=kw["transient_time"], h=kw["h"], eps=kw["eps"], idx1=idx1, idx2=idx2,
               r1lo=kw["param_lo"], r1hi=kw["param_hi"], r2lo=kw["param_lo_2"], r2hi=kw["param_hi_2"], data=v)
    assert_same_files(tmp_path, ["", "_config.csv"])


def test_ls2d_files_equal_reference_writer(eng, tmp_path):
    kw = dict(ic=(-10.0, -6.0, 0.0, 10.0), values=(0, 0.25, 0.05), param_index=1, param_index_2=2, param_lo=0.1,
              param_hi=0.35, param_lo_2=0.01, param_hi_2=0.1, h=0.01, transient_time=5.0, t_max=10.0, NT=0.1,
              eps=1e-6)
    req = ucb.Engine.ls2d_request(rk4_body(HYPER_ROSSLER), 4, kw["ic"], kw["values"], method=ucb.LS_FIXED, n_pts=5,
                                  csv_output_path=str(tmp_path / "eng.csv"), opt=ucb.options(**F32),
                                  **{k: v for k, v in kw.items() if k not in ("ic", "values")})
    v, f, _ = eng.run_ls2d(req)
    write_spec(tmp_path, "ls2d", n_pts=5, values=kw["values"], ic=kw["ic"], par_or_var=1, tMax=kw["t_max"],
               NT=kw["NT"], transient=kw["transient_time"], h=kw["h"], eps=kw["eps"], idx1=1, idx2=2, r1lo=0.1,
               r1hi=0.35, r2lo=0.01, r2hi=0.1, n_exp=4, data=np.ascontiguousarray(v.reshape(-1)))
    assert_same_files(tmp_path, ["", "_config.csv"])


def test_bif2d_files_equal_reference_writer(eng, tmp_path):
    req = ucb.Engine.bif2d_request(rk4_body(LORENZ), 3, (0.1, 0.1, 0.1), (0, 10.0, 28.0, 8 / 3), n_pts=6,
                                   param_index=2, param_index_2=1, param_lo=20.0, param_hi=200.0, param_lo_2=5.0,
                                   param_hi_2=15.0, h=0.01, transient_time=5.0, t_max=20.0, eps_dbscan=0.1,
                                   csv_output_path=str(tmp_path / "eng.csv"), opt=ucb.options(**F32))
    v, f, _ = eng.run_bif2d(req)
    write_spec(tmp_path, "bif2d", n_pts=6, values=(0, 10.0, 28.0, 8 / 3), ic=(0.1, 0.1, 0.1), par_or_var=1,
               tMax=20.0, transient=5.0, h=0.01, pre=1, eps_dbscan=0.1, writable_var=0, idx1=2, idx2=1, r1lo=20.0,
               r1hi=200.0, r2lo=5.0, r2hi=15.0, data=v)
    assert_same_files(tmp_path, ["", "_config.csv"])


@pytest.mark.parametrize("kind", ["lle1d", "ls1d"])
def test_1d_files_equal_reference_writer(eng, tmp_path, kind):
    kw = dict(n_pts=17, param_index=3, param_lo=2.0, param_hi=7.3, h=0.01, transient_time=5.0, t_max=10.0,
              NT=0.1, eps=1e-4)
    req = ucb.Engine.lle1d_request(rk4_body(ROSSLER), 3, (1.0, 1.0, 1.0), (0.0, 0.2, 0.2, 5.7),
                                   csv_output_path=str(tmp_path / "eng.csv"), opt=ucb.options(**F32), **kw)
    if kind == "lle1d":
        v, f, _ = eng.run_lle1d(req)
        extra = {}
    else:
        v, f, _ = eng.run_ls1d(req)
        v = np.ascontiguousarray(v.reshape(-1))
        extra = dict(n_exp=3)
    write_spec(tmp_path, kind, n_pts=17, values=(0.0, 0.2, 0.2, 5.7), ic=(1.0, 1.0, 1.0), tMax=10.0, NT=0.1,
               transient=5.0, h=0.01, eps=1e-4, idx1=3, lo=2.0, hi=7.3, data=v, **extra)
    assert_same_files(tmp_path, ["", "_config.csv"])


def test_bif1d_files_equal_reference_writer(eng, tmp_path):
    cap = 512
    req = ucb.Engine.bif1d_request(rk4_body(LORENZ), 3, (0.1, 0.1, 0.1), (0, 10.0, 28.0, 8 / 3), n_pts=24,
                                   param_index=2, param_lo=0.3, param_hi=200.0, h=0.01, transient_time=10.0,
                                   t_max=40.0, writable_var=0, max_peaks=cap,
                                   csv_output_path=str(tmp_path / "eng.csv"), opt=ucb.options(**F32))
    counts, peaks, intervals, _ = eng.run_bif1d(req)
    assert counts.max() < cap and (counts > 0).any() and (counts <= 0).any()
    write_spec(tmp_path, "bif1d", n_pts=24, values=(0, 10.0, 28.0, 8 / 3), ic=(0.1, 0.1, 0.1), tMax=40.0,
               transient=10.0, h=0.01, pre=1, writable_var=0, idx1=2, lo=0.3, hi=200.0, cap=cap,
               counts=counts.astype(np.int32), peaks=np.ascontiguousarray(peaks.reshape(-1)),
               intervals=np.ascontiguousarray(intervals.reshape(-1)))
    assert_same_files(tmp_path, ["", "_config.csv"])


def test_basins_files_equal_reference_writer(eng, tmp_path):
    from helpers import DUFFING
    req = ucb.Engine.basins_dbscan_request(rk4_body(DUFFING), 3, (0.0, 0.0, 0.0), (0.0,), n_pts=8, axis_x_lo=-2.5,
                                           axis_x_hi=2.5, axis_y_lo=-2.5, axis_y_hi=2.5, h=2 * np.pi / 200,
                                           t_max=100.0, transient_time=200.0, eps_dbscan=0.5,
                                           csv_output_path=str(tmp_path / "eng.csv"), opt=ucb.options(**F32))
    lab, f1, f2, cls, _ = eng.run_basins_dbscan(req)
    write_spec(tmp_path, "basins", n_pts=8, values=(0.0,), ic=(0.0, 0.0, 0.0), tMax=100.0, transient=200.0,
               h=2 * np.pi / 200, pre=1, eps_dbscan=0.5, writable_var=0, xvar=0, yvar=1, xlo=-2.5, xhi=2.5,
               ylo=-2.5, yhi=2.5, labels=lab.astype(np.int32), classes=cls.astype(np.int32), f1=f1, f2=f2)
    assert_same_files(tmp_path, ["", "_config.csv", "_1.csv", "_2.csv", "_3.csv"])
