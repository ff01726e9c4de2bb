"""Cancellation and progress during a run (the reference polls `cancel` and writes
`progress` between chunks, parametric_engine.h:85-92, parametric_engine.cpp:2780-2786).

Here one persistent kernel covers a whole map, so the engine mirrors the caller's cancel
word into a host-mapped control block while it waits: each warp checks it before taking
its next cells from the work queue (an adaptive DP5 cell also checks it every 4096 step
attempts), and the queue position is the progress. Nothing waits on the device; a warp
only stops taking work. The failure is made on the host: a Python thread sets the
caller's cancel word while the call runs (ctypes releases the GIL during the call)."""
import ctypes as C
import threading
import time

import numpy as np
import pytest

import ucb
from helpers import HYPER_ROSSLER, engine_request, lle2d_case, rk4_body

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    e = ucb.Engine(0)
    yield e
    e.close()


def run_watched(call, req, cancel_after_s=None):
    """Runs call(req) with cancel / progress words attached; a thread samples the progress
    every 2 ms and sets the cancel word after cancel_after_s. Returns (result or None,
    UcbError or None, seconds, progress samples)."""
    flag = C.c_int32(0)
    prog = C.c_float(-1.0)
    req.cancel = C.pointer(flag)
    req.progress = C.pointer(prog)
    seen = []
    done = threading.Event()

    def watch():
        t0 = time.perf_counter()
        while not done.is_set():
            seen.append(prog.value)
            if cancel_after_s is not None and time.perf_counter() - t0 >= cancel_after_s:
                flag.value = 1
            time.sleep(0.002)

    th = threading.Thread(target=watch)
    th.start()
    t0 = time.perf_counter()
    out, err = None, None
    try:
        out = call(req)
    except ucb.UcbError as ex:
        err = ex
    dt = time.perf_counter() - t0
    done.set()
    th.join()
    return out, err, dt, seen


def long_lle():
    # the headline map with a doubled horizon: 1024^2 cells, 2 x 10^5 measured steps each
    return lle2d_case(n=1024, t_max=2000.0, transient=100.0)


def test_progress_then_cancel_of_a_long_lle_map(eng):
    req = engine_request(ucb, long_lle(), precision=ucb.PREC_F64, mode=ucb.MODE_NATIVE)
    eng.run_lle2d(engine_request(ucb, lle2d_case(n=8, t_max=1.0, transient=1.0), precision=ucb.PREC_F64))
    out, err, full_s, seen = run_watched(eng.run_lle2d, req)
    assert err is None
    v_full, f_full, _ = out
    mid = [p for p in seen if 0.0 < p < 1.0]
    assert len(set(mid)) >= 3, seen[:50]                      # progress moved during the run
    assert all(b >= a - 0.2 for a, b in zip(mid, mid[1:]))   # and mostly forward
    assert req.progress.contents.value == 1.0
    out, err, cut_s, _ = run_watched(eng.run_lle2d, req, cancel_after_s=0.1)
    assert err is not None and err.code == ucb.UCB_E_CANCELLED, err
    assert cut_s < 0.5 * full_s, (cut_s, full_s)
    # the engine's control block is clear again: the next call runs to the end, same map
    req.cancel = None
    req.progress = None
    v, f, _ = eng.run_lle2d(req)
    np.testing.assert_array_equal(f, f_full)
    np.testing.assert_array_equal(v, v_full)


def test_cancel_of_a_long_dp5_spectrum_map(eng):
    # the spectrum configuration's window at 128^2 with t_end = 2e4: cells take up to the
    # 2e7-attempt cap (minutes for the map); a cancelled run abandons cells in flight
    req = ucb.Engine.ls2d_request(rk4_body(HYPER_ROSSLER), 4, (-10.0, -6.0, 0.0, 10.0), (0, 0.25, 0.05),
                                  method=ucb.LS_DP5, gs_every=10, rtol=1e-8, t_end=2e4, n_pts=128,
                                  param_index=1, param_index_2=2, param_lo=0.1, param_hi=0.35, param_lo_2=0.01,
                                  param_hi_2=0.1, h=0.01, transient_time=0.0, t_max=2e4, NT=1.0, eps=1e-6,
                                  opt=ucb.options(precision=ucb.PREC_F64))
    warm = ucb.Engine.ls2d_request(rk4_body(HYPER_ROSSLER), 4, (-10.0, -6.0, 0.0, 10.0), (0, 0.25, 0.05),
                                   method=ucb.LS_DP5, gs_every=10, rtol=1e-8, t_end=10.0, n_pts=4, param_index=1,
                                   param_index_2=2, param_lo=0.1, param_hi=0.35, param_lo_2=0.01, param_hi_2=0.1,
                                   h=0.01, t_max=10.0, NT=1.0, eps=1e-6, opt=ucb.options(precision=ucb.PREC_F64))
    eng.run_ls2d(warm)
    out, err, cut_s, _ = run_watched(eng.run_ls2d, req, cancel_after_s=0.2)
    assert err is not None and err.code == ucb.UCB_E_CANCELLED, err
    assert cut_s < 5.0, cut_s
    v, f, _ = eng.run_ls2d(warm)   # the engine runs the next map to the end
    assert (f != 0).all()
