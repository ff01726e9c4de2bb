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


@pytest.mark.parametrize("prec", [ucb.PREC_F64, ucb.PREC_F32])
def test_noalloc_matches_device_entry_twice(prec):
    torch = pytest.importorskip("torch")
    eng = ucb.Engine(0)
    c = lle2d_case(n=24, t_max=10.0, transient=5.0)
    req = engine_request(ucb, c, precision=prec, mode=ucb.MODE_NATIVE)
    cells = c["n_pts"] ** 2
    stream = torch.cuda.current_stream()
    ref_v = torch.empty(cells, dtype=torch.float64, device="cuda")
    ref_f = torch.empty(cells, dtype=torch.int32, device="cuda")
    eng.lle2d_device(req, ref_v.data_ptr(), ref_f.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    rv, rf = ref_v.cpu().numpy(), ref_f.cpu().numpy()
    eng.prepare_lle2d(req)
    for _ in range(2):
        v = torch.full((cells,), float("nan"), dtype=torch.float64, device="cuda")
        f = torch.zeros(cells, dtype=torch.int32, device="cuda")
        eng.lle2d_device_noalloc(req, v.data_ptr(), f.data_ptr(), stream.cuda_stream)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(f.cpu().numpy(), rf)
        np.testing.assert_allclose(v.cpu().numpy(), rv, rtol=1e-12, atol=0)
    eng.close()


def test_noalloc_rejects_oversize_and_unprepared():
    torch = pytest.importorskip("torch")
    eng = ucb.Engine(0)
    big = engine_request(ucb, lle2d_case(n=ucb_max() + 1))
    with pytest.raises(ucb.UcbError, match="scratch-array limit"):
        eng.lle2d_device_noalloc(big, 0, 0, 0)
    eng.close()


def ucb_max():
    return 4096
