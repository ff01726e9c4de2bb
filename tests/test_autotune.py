"""Launch-shape autotuning (ucb_autotune_*): the shape knobs compile for every kernel, bad
option values are rejected the reference's way, a search picks a shape that later runs
use, and no shape changes a single result bit."""
import numpy as np
import pytest

import ucb
from helpers import DUFFING, LORENZ, engine_request, lle2d_case, rk4_body

SHAPES = [dict(block_threads=256), dict(block_threads=64, unroll=4), dict(max_registers=64, unroll=2),
          dict(block_threads=512, max_registers=64)]


@pytest.mark.parametrize("shape", SHAPES)
def test_shapes_compile_for_every_kernel(shape):
    for prec, mode in ((ucb.PREC_F64, ucb.MODE_EXACT), (ucb.PREC_F32, ucb.MODE_NATIVE)):
        opt = dict(precision=prec, mode=mode, **shape)
        ucb.precompile(engine_request(ucb, lle2d_case(), **opt))
        # a system with a transcendental call (its packed FP32 pair form is emitted too)
        duffing = dict(lle2d_case(), body=rk4_body(DUFFING), ic=(0.0, 0.0, 0.0), values=(0.0,),
                       sweep_over_var=True, sweep_over_var_2=True, var_sweep_index=0, var_sweep_index_2=1,
                       param_lo=-1.0, param_hi=1.0, param_lo_2=-1.0, param_hi_2=1.0)
        for paired in (False, True):
            ucb.precompile(engine_request(ucb, duffing, paired_cells=paired, **opt))
        ucb.precompile(ucb.Engine.bif2d_request(rk4_body(LORENZ), 3, (0.1, 0.1, 0.1), (0, 10.0, 28.0, 8 / 3),
                                                n_pts=8, param_index=2, param_index_2=1, param_lo=20, param_hi=30,
                                                param_lo_2=5, param_hi_2=15, opt=ucb.options(**opt)))
        ucb.precompile(ucb.Engine.basins_request(rk4_body(DUFFING), 3, (0, 0, 0), (0.0,), n_pts=8, phase_var=2,
                                                 period=2 * np.pi, opt=ucb.options(**opt)))
        ucb.precompile(ucb.Engine.basins_dbscan_request(rk4_body(LORENZ), 3, (0, 0, 25.0), (0, 10.0, 10.0, 8 / 3),
                                                        n_pts=8, opt=ucb.options(**opt)))


@pytest.mark.parametrize("field,value,msg", [("block_threads", 48, "block_threads must be"),
                                             ("block_threads", 2048, "block_threads must be"),
                                             ("max_registers", 8, "max_registers must be"),
                                             ("unroll", 17, "unroll must be")])
def test_bad_shape_options_are_rejected(field, value, msg):
    with pytest.raises(ucb.UcbError, match=msg):
        ucb.precompile(engine_request(ucb, lle2d_case(), **{field: value}))


@pytest.mark.gpu
def test_autotune_lle2d_keeps_results_and_is_reused(tmp_path, monkeypatch):
    monkeypatch.setenv("UCB_TUNE_TABLE", str(tmp_path / "tuned.tsv"))
    c = lle2d_case(n=48, t_max=10.0, transient=5.0)
    eng = ucb.Engine(0)
    req = engine_request(ucb, c, precision=ucb.PREC_F64, mode=ucb.MODE_EXACT)
    ref, rflags, _ = eng.run_lle2d(req)
    rep = eng.autotune(req, force=True)
    assert rep["candidates"] >= 3 and rep["from_table"] == 0
    assert rep["block_threads"] in (64, 128, 256, 512) and rep["unroll"] in (1, 2, 4)
    assert rep["best_ms"] > 0 and rep["best_ms"] <= rep["default_ms"] and rep["registers"] > 0
    # the tuned shape is used by later runs and changes nothing
    vals, flags, _ = eng.run_lle2d(req)
    np.testing.assert_array_equal(vals, ref)
    np.testing.assert_array_equal(flags, rflags)
    for shape in SHAPES:
        v, _, _ = eng.run_lle2d(engine_request(ucb, c, precision=ucb.PREC_F64, mode=ucb.MODE_EXACT, **shape))
        np.testing.assert_array_equal(v, ref)
    eng.close()
    # a new engine finds the shape in the table
    eng2 = ucb.Engine(0)
    rep2 = eng2.autotune(req)
    assert rep2["from_table"] == 1 and rep2["key"] == rep["key"]
    assert (rep2["block_threads"], rep2["max_registers"], rep2["unroll"]) == \
        (rep["block_threads"], rep["max_registers"], rep["unroll"])
    eng2.close()


@pytest.mark.gpu
def test_autotune_basins_and_bif2d(tmp_path, monkeypatch):
    monkeypatch.setenv("UCB_TUNE_TABLE", str(tmp_path / "tuned.tsv"))
    eng = ucb.Engine(0)
    breq = ucb.Engine.basins_request(rk4_body(DUFFING), 3, (0.0, 0.0, 0.0), (0.0,), n_pts=32, axis_x_lo=-2.5,
                                     axis_x_hi=2.5, axis_y_lo=-2.5, axis_y_hi=2.5, period=2 * np.pi,
                                     steps_per_period=200, max_periods=60, phase_var=2,
                                     opt=ucb.options(precision=ucb.PREC_F64, mode=ucb.MODE_EXACT))
    ref = eng.run_basins(breq)[0]
    rep = eng.autotune(breq, force=True)
    assert rep["candidates"] >= 3
    np.testing.assert_array_equal(eng.run_basins(breq)[0], ref)
    b2 = ucb.Engine.bif2d_request(rk4_body(LORENZ), 3, (0.1, 0.1, 0.1), (0, 10.0, 28.0, 8 / 3), n_pts=24,
                                  param_index=2, param_index_2=1, param_lo=20.0, param_hi=200.0, param_lo_2=5.0,
                                  param_hi_2=15.0, h=0.01, transient_time=20.0, t_max=40.0, eps_dbscan=0.1,
                                  opt=ucb.options(precision=ucb.PREC_F64, mode=ucb.MODE_EXACT))
    ref2 = eng.run_bif2d(b2)[0]
    rep2 = eng.autotune(b2, force=True)
    assert rep2["candidates"] >= 3
    np.testing.assert_array_equal(eng.run_bif2d(b2)[0], ref2)
    eng.close()


def test_forced_system_compiles_in_every_form():
    """A system with a clock (a variable of constant derivative) gets the compensated FP32
    clock in the kernels whose Stepper serves one trajectory (tangent LLE, bifurcation,
    reference-method basins, DP5) and none in those that step several trajectories on one
    Stepper (shadow LLE, the fixed LS method): every combination compiles."""
    from helpers import DUFFING
    duffing = dict(lle2d_case(), body=rk4_body(DUFFING), ic=(0.0, 0.0, 0.0), values=(0.0,),
                   sweep_over_var=True, sweep_over_var_2=True, var_sweep_index=0, var_sweep_index_2=1,
                   param_lo=-1.0, param_hi=1.0, param_lo_2=-1.0, param_hi_2=1.0)
    body = rk4_body(DUFFING)
    grid = dict(n_pts=4, sweep_over_var=True, sweep_over_var_2=True, var_sweep_index=0, var_sweep_index_2=1,
                param_lo=-1, param_hi=1, param_lo_2=-1, param_hi_2=1)
    for prec in (ucb.PREC_F32, ucb.PREC_F64):
        opt = ucb.options(precision=prec)
        for method in (ucb.LLE_AUTO, ucb.LLE_SHADOW):
            ucb.precompile(engine_request(ucb, duffing, precision=prec, lle_method=method))
        ucb.precompile(ucb.Engine.ls2d_request(body, 3, (0.0, 0.0, 0.0), (0.0,), method=ucb.LS_DP5, t_end=10.0,
                                               t_max=10.0, opt=opt, **grid))
        ucb.precompile(ucb.Engine.ls2d_request(body, 3, (0.0, 0.0, 0.0), (0.0,), method=ucb.LS_FIXED, t_max=10.0,
                                               opt=opt, **grid))
        ucb.precompile(ucb.Engine.bif2d_request(body, 3, (0.0, 0.0, 0.0), (0.0,), opt=opt, **grid))
        ucb.precompile(ucb.Engine.basins_dbscan_request(body, 3, (0, 0, 0), (0.0,), n_pts=4, opt=opt))
        ucb.precompile(ucb.Engine.bif1d_request(body, 3, (0.0, 0.0, 0.0), (0.0,), n_pts=4, sweep_over_var=True,
                                                var_sweep_index=0, param_lo=-1, param_hi=1, opt=opt))


def test_register_cap_reaches_the_compiled_kernel(tmp_path):
    """A register cap changes the build: the DP5 spectrum kernel (about 250 registers
    uncapped in FP64) is compiled within a 128-register cap. Checked on the compiler's own
    report, in a child process with a fresh CUBIN cache."""
    import re
    import subprocess
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    code = f"""
import sys
sys.path.insert(0, {str(root / 'u-cuda_b200')!r}); sys.path.insert(0, {str(root / 'tests')!r})
import ucb
from helpers import HYPER_ROSSLER, rk4_body
cap = int(sys.argv[1])
ucb.precompile(ucb.Engine.ls2d_request(rk4_body(HYPER_ROSSLER), 4, (-10.0, -6.0, 0.0, 10.0), (0, 0.25, 0.05),
                                       method=ucb.LS_DP5, t_end=10.0, n_pts=4, param_index=1, param_index_2=2,
                                       param_lo=0.1, param_hi=0.35, param_lo_2=0.01, param_hi_2=0.1, t_max=10.0,
                                       opt=ucb.options(precision=ucb.PREC_F64, max_registers=cap)))
"""
    used = {}
    for cap in (0, 128):
        env = dict(__import__("os").environ, UCB_PTXAS_VERBOSE="1", UCB_CUBIN_CACHE=str(tmp_path / f"c{cap}"))
        r = subprocess.run([sys.executable, "-c", code, str(cap)], env=env, capture_output=True, text=True,
                           timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        regs = [int(m) for m in re.findall(r"Used (\d+) registers", r.stderr)]
        assert regs, r.stderr[-2000:]
        used[cap] = max(regs)
    assert used[0] > 128 and used[128] <= 128
