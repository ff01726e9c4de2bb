"""Surrogate MLP: the CPU oracle is pinned by finite differences; the GPU training kernels
(tcgen05 GEMMs, loss, GELU backward) are checked against it; training reduces the loss on
a known function; the surrogate-refined map is checked against the full plain map."""
import ctypes as C
import time

import numpy as np
import pytest

from oracle import mlp_oracle as MO

FOURIER, HIDDEN, LAYERS = 64, 128, 2


def _rand_params(rng, fourier, hidden, layers, scale=1.0):
    p = []
    for o, i in MO.layer_shapes(fourier, hidden, layers):
        p.append(rng.normal(0, scale * np.sqrt(2.0 / i), size=o * i))
        p.append(rng.normal(0, 0.1, size=o))
    return np.concatenate(p)


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = _rand_params(rng, 4, 8, 2)
    # the flat layout here uses fourier=4 / hidden=8 (the oracle has no size rules)
    B = rng.normal(0, 2.0, size=(4, 2))
    u = rng.uniform(size=(20, 2))
    y = rng.normal(size=20)
    loss, g = MO.loss_and_grad(p, B, u, y, 8, 2, beta=0.5, y_mean=0.1, y_std=1.3, bf16=False)
    # beta weight is a constant in the loss: finite differences of the weighted loss with
    # the weight frozen at p
    out0, _ = MO.forward(p, B, u, 8, 2, bf16=False)
    w = np.exp(0.5 * np.clip(out0[:, 1], -16, 16))

    def frozen_loss(q):
        out, _ = MO.forward(q, B, u, 8, 2, bf16=False)
        ys = (y - 0.1) / 1.3
        lv = np.clip(out[:, 1], -16, 16)
        return float(np.sum(w * 0.5 * (lv + (out[:, 0] - ys) ** 2 * np.exp(-lv))) / len(y))

    assert abs(frozen_loss(p) - loss) < 1e-12
    idx = rng.choice(len(p), size=60, replace=False)
    for i in idx:
        e = np.zeros_like(p)
        e[i] = 1e-6
        fd = (frozen_loss(p + e) - frozen_loss(p - e)) / 2e-6
        assert abs(fd - g[i]) < 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, 1.0078125, -2.5, 3.0e-3], dtype=np.float32)
    r = MO.bf16_round(x)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: even -> 1; 1 + 1.5 * 2^-8 rounds up
    assert list(r[:4]) == [1.0, 1.0, 1.0078125, 1.0078125]
    assert r[4] == -2.5
    assert abs(r[5] - 3.0e-3) / 3.0e-3 < 2 ** -8


# --------------------------------------------------------------------------- GPU
@pytest.fixture(scope="module")
def ucb_engine():
    import ucb
    e = ucb.Engine(0)
    yield e
    e.close()


def _net(ucb, eng, **kw):
    cfg = dict(fourier=FOURIER, hidden=HIDDEN, layers=LAYERS, fourier_scale=3.0, seed=7, batch=1024,
               train_steps=300, lr=3e-3, lr_final=1e-4, beta_nll=0.5)
    cfg.update(kw)
    return ucb.Mlp(eng, **cfg)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1000, 4096])
def test_gpu_gradient_matches_oracle(ucb_engine, n):
    import ucb
    net = _net(ucb, ucb_engine)
    rng = np.random.default_rng(n)
    u = rng.uniform(size=(n, 2)).astype(np.float32)
    y = (np.sin(5 * u[:, 0]) * np.cos(3 * u[:, 1]) + 0.1 * rng.normal(size=n)).astype(np.float32)
    net.set_target_scale(0.05, 0.7)
    p = net.get_params()
    B = net.fourier()
    loss, g = net.loss_grad(u, y)
    lo, go = MO.loss_and_grad(p, B, u, y, HIDDEN, LAYERS, beta=0.5, y_mean=0.05, y_std=0.7, bf16=True)
    assert abs(loss - lo) <= 2e-3 * abs(lo) + 1e-6
    off = 0
    for l, (o, i) in enumerate(MO.layer_shapes(FOURIER, HIDDEN, LAYERS)):
        for name, size in (("W", o * i), ("b", o)):
            a, b = g[off:off + size].astype(np.float64), go[off:off + size]
            off += size
            rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
            cos = float(a @ b / max(np.linalg.norm(a) * np.linalg.norm(b), 1e-30))
            assert rel < 2e-2 and cos > 0.9995, (l, name, rel, cos)


@pytest.mark.gpu
def test_gpu_prediction_matches_oracle(ucb_engine):
    import torch
    import ucb
    net = _net(ucb, ucb_engine)
    rng = np.random.default_rng(3)
    n = 3000
    u = rng.uniform(size=(n, 2)).astype(np.float32)
    net.set_target_scale(-0.2, 2.0)
    du = torch.from_numpy(u).cuda()
    dm = torch.empty(n, device="cuda")
    ds = torch.empty(n, device="cuda")
    net.predict(du.data_ptr(), n, dm.data_ptr(), ds.data_ptr())
    torch.cuda.synchronize()
    m_ref, s_ref = MO.predict(net.get_params(), net.fourier(), u, HIDDEN, LAYERS, y_mean=-0.2, y_std=2.0)
    m, s = dm.cpu().numpy(), ds.cpu().numpy()
    # BF16 rounding flips of single activations (GPU FP32 vs oracle float64 sums) move a
    # row by ~1e-3 of the output scale at most
    scale = np.abs(m_ref).max()
    assert np.max(np.abs(m - m_ref)) < 1e-2 * scale + 1e-5
    assert np.mean(np.abs(m - m_ref)) < 1e-3 * scale + 1e-6
    assert np.max(np.abs(s / s_ref - 1)) < 1e-2


@pytest.mark.gpu
def test_gpu_layer_by_layer_path_matches_oracle(ucb_engine):
    """A hidden width the fused kernels do not cover (384) runs the features kernel and one
    GEMM per layer, for training and prediction alike: gradients and predictions against
    the oracle."""
    import torch
    import ucb
    hidden, layers = 384, 2
    net = ucb.Mlp(ucb_engine, fourier=FOURIER, hidden=hidden, layers=layers, fourier_scale=3.0, seed=5, batch=1024,
                  train_steps=1)
    rng = np.random.default_rng(21)
    net.set_params(_rand_params(rng, FOURIER, hidden, layers).astype(np.float32))
    n = 2000
    u = rng.uniform(size=(n, 2)).astype(np.float32)
    y = (np.sin(4 * u[:, 0]) + 0.1 * rng.normal(size=n)).astype(np.float32)
    net.set_target_scale(0.1, 0.8)
    p = net.get_params()
    B = net.fourier()
    loss, g = net.loss_grad(u, y)
    lo, go = MO.loss_and_grad(p, B, u, y, hidden, layers, beta=0.5, y_mean=0.1, y_std=0.8, bf16=True)
    assert abs(loss - lo) <= 2e-3 * abs(lo) + 1e-6
    rel = np.linalg.norm(g - go) / np.linalg.norm(go)
    assert rel < 2e-2, rel
    du = torch.from_numpy(u).cuda()
    dm = torch.empty(n, device="cuda")
    ds = torch.empty(n, device="cuda")
    net.predict(du.data_ptr(), n, dm.data_ptr(), ds.data_ptr())
    torch.cuda.synchronize()
    m_ref, s_ref = MO.predict(p, B, u, hidden, layers, y_mean=0.1, y_std=0.8)
    scale = np.abs(m_ref).max()
    assert np.max(np.abs(dm.cpu().numpy() - m_ref)) < 1e-2 * scale + 1e-5
    assert np.max(np.abs(ds.cpu().numpy() / s_ref - 1)) < 1e-2
    net.close()


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 127, 129, 40000])
def test_gpu_fused_prediction_matches_oracle_at_the_surrogate_size(ucb_engine, n):
    """The fused prediction kernel (features, hidden layers and output of a 128-row tile in
    one CTA, activations in shared memory) on the surrogate's network (64 Fourier features,
    4 x 256 GELU): ragged row counts, and at 40,000 rows (313 tiles) every CTA runs a second
    pair of tiles with one slot empty at the end."""
    import torch
    import ucb
    net = ucb.Mlp(ucb_engine, fourier=64, hidden=256, layers=4, fourier_scale=2.0, seed=11, batch=1024,
                  train_steps=1)
    rng = np.random.default_rng(n)
    p = _rand_params(rng, 64, 256, 4, scale=0.8)
    net.set_params(p.astype(np.float32))
    net.set_target_scale(0.3, 1.5)
    u = rng.uniform(size=(n, 2)).astype(np.float32)
    du = torch.from_numpy(u).cuda()
    dm = torch.full((n + 1,), 7.0, device="cuda")
    ds = torch.full((n + 1,), 7.0, device="cuda")
    net.predict(du.data_ptr(), n, dm.data_ptr(), ds.data_ptr())
    torch.cuda.synchronize()
    m_ref, s_ref = MO.predict(net.get_params(), net.fourier(), u, 256, 4, y_mean=0.3, y_std=1.5)
    m, s = dm.cpu().numpy(), ds.cpu().numpy()
    assert m[n] == 7.0 and s[n] == 7.0  # nothing written past the last row
    scale = np.abs(m_ref).max()
    assert np.max(np.abs(m[:n] - m_ref)) < 1e-2 * scale + 1e-5
    assert np.mean(np.abs(m[:n] - m_ref)) < 1e-3 * scale + 1e-6
    assert np.max(np.abs(s[:n] / s_ref - 1)) < 1e-2
    net.close()


@pytest.mark.gpu
def test_gpu_training_fits_smooth_function(ucb_engine):
    import torch
    import ucb
    net = _net(ucb, ucb_engine, fourier=64, hidden=256, layers=4, batch=4096, train_steps=1500, lr=2e-3,
               lr_final=2e-5, fourier_scale=2.0)
    rng = np.random.default_rng(11)
    n = 16384
    u = rng.uniform(size=(n, 2)).astype(np.float32)
    f = lambda v: np.sin(4 * v[:, 0]) * np.cos(3 * v[:, 1]) + 0.5 * v[:, 0] ** 2
    y = f(u).astype(np.float32)
    du = torch.from_numpy(u).cuda()
    dy = torch.from_numpy(y).cuda()
    net.fit(du.data_ptr(), dy.data_ptr(), n)
    ut = rng.uniform(size=(8192, 2)).astype(np.float32)
    dut = torch.from_numpy(ut).cuda()
    dm = torch.empty(len(ut), device="cuda")
    ds = torch.empty(len(ut), device="cuda")
    net.predict(dut.data_ptr(), len(ut), dm.data_ptr(), ds.data_ptr())
    torch.cuda.synchronize()
    err = np.abs(dm.cpu().numpy() - f(ut))
    print("rmse / std", np.sqrt(np.mean(err ** 2)) / np.std(f(ut)), "median sd / std",
          np.median(ds.cpu().numpy()) / np.std(f(ut)))
    assert np.sqrt(np.mean(err ** 2)) < 0.02 * np.std(f(ut)), np.sqrt(np.mean(err ** 2))
    # the network's own uncertainty is calibrated to the residual scale
    assert np.median(ds.cpu().numpy()) < 0.05 * np.std(f(ut))


def test_mlp_config_validation():
    import ucb
    eng = ucb.Engine(0)
    with pytest.raises(ucb.UcbError, match="invalid MLP configuration"):
        ucb.Mlp(eng, fourier=33)
    with pytest.raises(ucb.UcbError, match="invalid MLP configuration"):
        ucb.Mlp(eng, batch=1000)
    eng.close()


def _lorenz_stable_case(n, t_max=4000.0):
    """Lorenz LLE map over sigma in [4, 16] x rho in [0.2, 0.9]: the origin is a stable node
    there, so the exponent is a smooth function of the parameters up to a per-cell probe
    term log|c1| / t_max, c1 the random probe direction's component along the slowest
    eigenvector (uniform on [-1, 1] in three dimensions). A smooth predictor misses a cell by
    more than 2e-3 when |log|c1| + 1| > 2e-3 t_max: on 0.7 % of the cells at t_max = 2000,
    on 0.01 % at t_max = 4000, which lets a 99.5 % coverage be certified."""
    from helpers import rk4_body, LORENZ
    return dict(body=rk4_body(LORENZ), nx=3, ic=(0.5, 0.5, 0.5), values=(0.0, 10.0, 0.5, 8.0 / 3.0), n_pts=n,
                param_index=1, param_index_2=2, param_lo=4.0, param_hi=16.0, param_lo_2=0.2, param_hi_2=0.9,
                h=0.01, transient_time=10.0, t_max=t_max, NT=0.1, eps=1e-4, max_value=1e6)


def _full_map(ucb_engine, c, prec):
    import torch
    import ucb
    from helpers import engine_request
    n = c["n_pts"]
    v = torch.empty(n * n, dtype=torch.float64, device="cuda")
    f = torch.empty(n * n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ucb_engine.lle2d_device(engine_request(ucb, c, precision=prec), v.data_ptr(), f.data_ptr(), 0)
    torch.cuda.synchronize()
    ms = (time.perf_counter() - t0) * 1e3
    return v.cpu().numpy(), f.cpu().numpy(), ms


def _surrogate(ucb_engine, c, **kw):
    import torch
    import ucb
    from helpers import engine_request
    n = c["n_pts"]
    req = ucb.surrogate_request(engine_request(ucb, c, precision=ucb.PREC_F32), **kw)
    v = torch.empty(n * n, dtype=torch.float64, device="cuda")
    f = torch.empty(n * n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    res = ucb_engine.run_lle2d_surrogate(req, v.data_ptr(), f.data_ptr(), 0)
    torch.cuda.synchronize()
    ms = (time.perf_counter() - t0) * 1e3
    return v.cpu().numpy(), f.cpu().numpy(), res, ms


LORENZ_NET = dict(batch=1024, train_steps=1500, fourier_scale=1.0, seed=3)


@pytest.mark.gpu
def test_surrogate_map_gain_and_calibrated_error(ucb_engine):
    """What the trained network gains: on a map with smooth regions it vouches for a large
    share of the cells, so only the samples and the rest are integrated, and the cells it
    predicts are within the calibrated tolerance (2e-3 on 99.5 % of them) of the full plain
    (FP64) map. Training is reproducible (split-K partial tiles and per-block sums are added
    in a fixed order), so a second call gives the same map bit for bit."""
    import ucb
    c = _lorenz_stable_case(256)
    ref64, f64, _ = _full_map(ucb_engine, c, ucb.PREC_F64)
    ref32, _, _ = _full_map(ucb_engine, c, ucb.PREC_F32)
    assert (f64 == 1).all()
    kw = dict(train_pts=64, tol=2e-3, coverage=0.995, lle_band=0.0, mlp=LORENZ_NET)
    vals, flags, res, _ = _surrogate(ucb_engine, c, **kw)
    vals2, flags2, res2, _ = _surrogate(ucb_engine, c, **kw)
    np.testing.assert_array_equal(flags2, flags)
    np.testing.assert_array_equal(vals2, vals)
    assert res.gated == 0 and res.pilot_predictable >= 0.05
    assert res.n_samples == 64 * 64 and res.n_samples + res.n_refined + res.n_predicted == 256 * 256
    assert set(np.unique(flags)) <= {1, 2}
    pred = flags == 2
    print("predicted", pred.mean(), "threshold", res.sigma_threshold, "calibration", res.calib_within_tol,
          "pilot share", res.pilot_predictable, "train ms", res.train_ms)
    # the gain: at least half of the map is not integrated
    assert pred.mean() >= 0.5, pred.mean()
    err = np.abs(vals[pred] - ref64[pred])
    assert (err <= 2e-3).mean() >= 0.995, ((err <= 2e-3).mean(), err.max())
    # integrated cells: samples carry the FP64 value, re-integrated cells the FP32 value
    integ = flags == 1
    is64 = vals[integ] == ref64[integ]
    is32 = vals[integ] == ref32[integ]
    assert (is64 | is32).all()
    assert is64.sum() >= res.n_samples - 1


@pytest.mark.gpu
def test_surrogate_wall_clock_gain_over_the_fp32_map(ucb_engine):
    """The same smooth map at 1024^2 with t_max = 4000: the surrogate-refined call (samples,
    training on this GPU, prediction, re-integration of the rest) takes less wall-clock time
    than integrating the whole map in the FP32 form, and its predicted cells keep the 2e-3
    tolerance against the FP64 map on 99.5 % of them."""
    import ucb
    c = _lorenz_stable_case(1024)
    ref64, _, _ = _full_map(ucb_engine, c, ucb.PREC_F64)
    _full_map(ucb_engine, c, ucb.PREC_F32)  # compiled and warm
    _, _, ms32 = _full_map(ucb_engine, c, ucb.PREC_F32)
    kw = dict(train_pts=256, tol=2e-3, coverage=0.995, lle_band=0.0, mlp=LORENZ_NET)
    _surrogate(ucb_engine, c, **kw)  # network buffers and the captured training step exist
    vals, flags, res, ms = _surrogate(ucb_engine, c, **kw)
    pred = flags == 2
    print(f"surrogate {ms:.0f} ms vs FP32 map {ms32:.0f} ms; predicted {pred.mean():.3f}, "
          f"pilot share {res.pilot_predictable:.3f}, train {res.train_ms:.0f} ms")
    assert res.gated == 0
    assert ms < ms32, (ms, ms32)
    err = np.abs(vals[pred] - ref64[pred])
    assert (err <= 2e-3).mean() >= 0.995, ((err <= 2e-3).mean(), err.max())


@pytest.mark.gpu
def test_surrogate_gate_skips_training_on_a_chaotic_map(ucb_engine):
    """On the chaotic Rossler map no smooth predictor can vouch for cells at 2e-3 / 99.5 %:
    the pilot samples show it before any training, so no network is trained and every other
    cell is integrated in the FP32 form (the call costs the FP32 map plus the pilot)."""
    import ucb
    from helpers import lle2d_case
    c = lle2d_case(n=256, t_max=200.0, transient=50.0)
    ref64, _, _ = _full_map(ucb_engine, c, ucb.PREC_F64)
    ref32, _, _ = _full_map(ucb_engine, c, ucb.PREC_F32)
    vals, flags, res, _ = _surrogate(ucb_engine, c, train_pts=64, tol=2e-3, coverage=0.995, lle_band=0.05)
    assert res.gated == 1 and res.pilot_predictable < 0.05
    assert res.n_predicted == 0 and res.train_ms < 1.0
    assert not (flags == 2).any()
    pilots = vals == ref64
    assert pilots.sum() >= res.n_samples - 1
    np.testing.assert_array_equal(vals[~pilots], ref32[~pilots])
