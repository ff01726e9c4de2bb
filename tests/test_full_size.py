"""The benchmark map at its full size (Rossler LLE, 1024 x 1024 cells over b in [0.05, 2] x
c in [2, 20], RK4 h = 0.01, 1e4 transient + 1e5 measured steps, renormalised every 10
steps): parity with the oracle on a seeded sample of cells, and properties that hold at any
size — a cell's value does not depend on which launch computes it (full map, cell list,
another precision's work queue order), the sentinels never appear in this window, and the
FP32 tangent form agrees with FP64 on the contracting cells, whose exponent is
well-conditioned."""
import numpy as np
import pytest

from oracle import oracle as O
import ucb
from helpers import engine_request, kernel_grid, lle2d_case

N = 1024


def full_case():
    return lle2d_case(n=N, t_max=1000.0, transient=100.0)


def sample_cells(count, seed):
    """Seeded sample of distinct cells over the whole map (kernel = user order here)."""
    return np.sort(np.random.default_rng(seed).choice(N * N, size=count, replace=False))


@pytest.fixture(scope="module")
def eng():
    e = ucb.Engine(0)
    yield e
    e.close()


@pytest.fixture(scope="module")
def exact_map(eng):
    v, f, _ = eng.run_lle2d(engine_request(ucb, full_case(), precision=ucb.PREC_F64, mode=ucb.MODE_EXACT))
    return v, f


@pytest.mark.gpu
def test_full_map_exact_form_equals_oracle_on_sampled_cells(exact_map):
    v, f = exact_map
    assert (f == 1).all()
    cells = sample_cells(256, seed=11)
    c = full_case()
    ov, of = O.lle2d(O.Krs(c["body"], 3), kernel_grid(c), cells=cells)
    np.testing.assert_array_equal(f[cells], of)
    # trajectories are bit-identical; the block logs differ by device vs host log (<= 1 ulp)
    np.testing.assert_allclose(v[cells], ov, rtol=1e-12, atol=1e-15)


@pytest.mark.gpu
def test_cell_list_equals_full_map(eng):
    """The cell-list entry (held-out subsets, re-integration) returns the full map's values
    bit for bit, for both precisions."""
    import torch
    cells = sample_cells(4096, seed=5)
    d_cells = torch.from_numpy(cells).cuda()
    for prec in (ucb.PREC_F64, ucb.PREC_F32):
        req = engine_request(ucb, full_case(), precision=prec, mode=ucb.MODE_NATIVE)
        full, flags, _ = eng.run_lle2d(req)
        jv = torch.empty(len(cells), dtype=torch.float64, device="cuda")
        jf = torch.empty(len(cells), dtype=torch.int32, device="cuda")
        eng.lle2d_cells(req, d_cells.data_ptr(), len(cells), jv.data_ptr(), jf.data_ptr(), 0)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(jv.cpu().numpy(), full[cells])
        np.testing.assert_array_equal(jf.cpu().numpy(), flags[cells])


@pytest.mark.gpu
def test_fp32_tangent_form_agrees_on_contracting_cells(eng, exact_map):
    ref, _ = exact_map
    v32, f32, _ = eng.run_lle2d(engine_request(ucb, full_case(), precision=ucb.PREC_F32, mode=ucb.MODE_NATIVE))
    assert (f32 == 1).all() and np.isfinite(v32).all()
    stable = ref < -0.02   # a stable fixed point or cycle: the exponent is a smooth function of the cell
    assert stable.sum() > 1000
    d = np.abs(v32[stable] - ref[stable])
    assert (d <= 2e-3).mean() >= 0.995
    # over the whole map: the same regime picture (sign of the exponent beyond the noise band)
    chaotic = ref > 0.02
    assert ((v32 > 0.01) == chaotic)[chaotic | stable].mean() >= 0.99
