"""The allocation-free LLE entry point (ucb_lle2d_device_noalloc) against the existing
device entry point (ucb_lle2d_device), through the C ABI.

It exists for callers that cannot allocate device memory themselves: programs that own
all device memory through their own pool or a fixed budget, and time-critical loops that
must not call cudaMalloc / cudaFree. Its scratch lives in a fixed array inside the
library, shared by every call. Both entry points run the same kernel on the same inputs,
so the results must be identical; two calls in a row check that each call resets the
shared scratch it depends on. This file is named to be collected last."""
import numpy as np
import pytest

import ucb
from helpers import engine_request, lle2d_case

pytestmark = pytest.mark.gpu

MAX_PTS = 4096  # UCB_NOALLOC_MAX_PTS


def reference_map(req, cells, torch):
    """The map through the existing device entry point, on an engine of its own."""
    eng = ucb.Engine(0)
    v = torch.empty(cells, dtype=torch.float64, device="cuda")
    f = torch.empty(cells, dtype=torch.int32, device="cuda")
    eng.lle2d_device(req, v.data_ptr(), f.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    eng.close()
    return v.cpu().numpy(), f.cpu().numpy()


@pytest.mark.parametrize("prec", [ucb.PREC_F64, ucb.PREC_F32])
def test_noalloc_matches_device_entry_twice(prec):
    torch = pytest.importorskip("torch")
    c = lle2d_case(n=24, t_max=10.0, transient=5.0)
    req = engine_request(ucb, c, precision=prec, mode=ucb.MODE_NATIVE)
    cells = c["n_pts"] ** 2
    rv, rf = reference_map(req, cells, torch)
    # a fresh engine on which only the set-up call has run
    eng = ucb.Engine(0)
    eng.prepare_lle2d(req)
    stream = torch.cuda.current_stream()
    for _ in range(2):
        v = torch.full((cells,), float("nan"), dtype=torch.float64, device="cuda")
        f = torch.zeros(cells, dtype=torch.int32, device="cuda")
        eng.lle2d_device_noalloc(req, v.data_ptr(), f.data_ptr(), stream.cuda_stream)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(f.cpu().numpy(), rf)
        np.testing.assert_allclose(v.cpu().numpy(), rv, rtol=1e-12, atol=0)
    eng.close()


def test_noalloc_allocates_no_device_memory():
    torch = pytest.importorskip("torch")
    c = lle2d_case(n=64, t_max=10.0, transient=5.0)
    req = engine_request(ucb, c, precision=ucb.PREC_F32, mode=ucb.MODE_NATIVE)
    cells = c["n_pts"] ** 2
    eng = ucb.Engine(0)
    eng.prepare_lle2d(req)
    v = torch.empty(cells, dtype=torch.float64, device="cuda")
    f = torch.empty(cells, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    eng.lle2d_device_noalloc(req, v.data_ptr(), f.data_ptr(), stream)   # first launch of the kernel
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        eng.lle2d_device_noalloc(req, v.data_ptr(), f.data_ptr(), stream)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    eng.close()


def test_noalloc_rejects_an_unprepared_engine():
    torch = pytest.importorskip("torch")
    req = engine_request(ucb, lle2d_case(n=8, t_max=2.0, transient=1.0))
    v = torch.empty(64, dtype=torch.float64, device="cuda")
    f = torch.empty(64, dtype=torch.int32, device="cuda")
    eng = ucb.Engine(0)
    with pytest.raises(ucb.UcbError, match="not prepared"):
        eng.lle2d_device_noalloc(req, v.data_ptr(), f.data_ptr(), 0)
    # prepared for another request (other precision: another kernel) is still unprepared
    eng.prepare_lle2d(engine_request(ucb, lle2d_case(n=8, t_max=2.0, transient=1.0), precision=ucb.PREC_F32))
    with pytest.raises(ucb.UcbError, match="not prepared"):
        eng.lle2d_device_noalloc(req, v.data_ptr(), f.data_ptr(), 0)
    eng.close()


def test_noalloc_rejects_oversize():
    eng = ucb.Engine(0)
    big = engine_request(ucb, lle2d_case(n=MAX_PTS + 1))
    with pytest.raises(ucb.UcbError, match="scratch-array limit"):
        eng.lle2d_device_noalloc(big, 0, 0, 0)
    eng.close()
