"""Basins of attraction by the reference's own method (run_basins / run_basins_recluster):
per initial-condition cell a class (1 oscillating, -1 fixed point, 0 unbound) and two
features of the peaks, then DBSCAN of the features.

The exact form integrates bit-identically to the oracle, so classes and features equal
the oracle's cell for cell and the labels must too. The clustering is checked on its own
(run_basins_recluster) against the oracle's literal restatement of the reference's host
loop on synthetic features built to hit its cases: chains through many grid squares,
square pairs with thousands of cells each that are just within / just beyond eps,
duplicates, non-finite features, fixed points and oscillating cells in one cluster, class
values that never seed. At 1M cells, where the literal loop is too slow, it is checked
against the component rule that loop implies (proved equal to it on small inputs here on
the CPU)."""
import math

import numpy as np
import pytest

import ucb
from helpers import DUFFING, LORENZ, rk4_body
from oracle import oracle as O


def lorenz_case(**kw):
    """Lorenz rho = 10: every trajectory settles on C+ or C- (two fixed-point basins)."""
    d = dict(body=LORENZ, nx=3, n_pts=16, axis_x_var=0, axis_y_var=1, axis_x_lo=-20.0, axis_x_hi=20.0,
             axis_y_lo=-20.0, axis_y_hi=20.0, ic=(0.0, 0.0, 25.0), values=(0, 10.0, 10.0, 8 / 3), h=0.01,
             transient_time=100.0, t_max=20.0, max_value=1e6, eps_dbscan=0.5, writable_var=0, pre_scaller=1,
             feature1=0, feature2=1, mult1=1.0, mult2=1.0)
    d.update(kw)
    return d


CASES = {
    "fixed_points": lorenz_case(),
    "chaotic": lorenz_case(values=(0, 10.0, 28.0, 8 / 3), transient_time=50.0),
    "unbound": lorenz_case(axis_x_lo=-80.0, axis_x_hi=80.0, axis_y_lo=-80.0, axis_y_hi=80.0, max_value=60.0),
    "features": lorenz_case(values=(0, 10.0, 28.0, 8 / 3), transient_time=20.0, feature1=4, feature2=7, mult1=2.0,
                            mult2=0.5, writable_var=-1, pre_scaller=2, eps_dbscan=0.05),
    "duffing": dict(body=DUFFING, nx=3, n_pts=16, axis_x_var=0, axis_y_var=1, axis_x_lo=-2.5, axis_x_hi=2.5,
                    axis_y_lo=-2.5, axis_y_hi=2.5, ic=(0.0, 0.0, 0.0), values=(0.0,), h=2 * math.pi / 200,
                    transient_time=60.0, t_max=30.0, max_value=1e6, eps_dbscan=0.05, writable_var=0,
                    pre_scaller=1, feature1=0, feature2=1, mult1=1.0, mult2=1.0),
}

KEYS = ("n_pts", "axis_x_var", "axis_y_var", "axis_x_lo", "axis_x_hi", "axis_y_lo", "axis_y_hi", "writable_var", "h",
        "t_max", "transient_time", "pre_scaller", "max_value", "eps_dbscan", "feature1", "feature2", "mult1", "mult2")


def request(c, **opt):
    return ucb.Engine.basins_dbscan_request(rk4_body(c["body"]), c["nx"], c["ic"], c["values"],
                                            csv_output_path=c.get("csv"), opt=ucb.options(**opt),
                                            **{k: c[k] for k in KEYS if k in c})


def oracle(c, numb="f64"):
    return O.basins_ref(O.Krs(rk4_body(c["body"]), c["nx"], numb), c)


# ------------------------------------------------------------------------------ CPU


def test_basins_dbscan_validation_messages():
    eng = ucb.Engine(0)
    for field, value, msg in (("eps_dbscan", 0.0, "eps_dbscan must be > 0"),
                              ("pre_scaller", 0, "pre_scaller must be > 0"),
                              ("writable_var", 3, "writable_var out of range"),
                              ("axis_y_var", 0, "axis_x_var == axis_y_var"),
                              ("axis_x_var", 3, "axis_x_var out of range"),
                              ("n_pts", 0, "n_pts must be > 0"),
                              ("transient_time", -1.0, "transient_time must be >= 0")):
        with pytest.raises(ucb.UcbError, match=msg):
            eng.run_basins_dbscan(request(lorenz_case(**{field: value})))
    with pytest.raises(ucb.UcbError, match="amountOfPointsInBlock"):
        eng.run_basins_dbscan(request(lorenz_case(t_max=0.005)))
    f = np.zeros(4)
    with pytest.raises(ucb.UcbError, match="eps_dbscan must be > 0"):
        eng.run_basins_recluster("x", 3, 2, 0.0, f, f, np.ones(4))
    with pytest.raises(ucb.UcbError, match="krs_body is empty"):
        eng.run_basins_recluster("", 3, 2, 0.5, f, f, np.ones(4))
    eng.close()


@pytest.mark.parametrize("prec,mode", [(ucb.PREC_F64, ucb.MODE_EXACT), (ucb.PREC_F32, ucb.MODE_EXACT),
                                       (ucb.PREC_F64, ucb.MODE_NATIVE)])
def test_basins_dbscan_kernel_compiles_for_sm100a(prec, mode):
    ucb.precompile_lle2d(request(CASES["features"], precision=prec, mode=mode))


def test_oracle_lorenz_fixed_point_basins():
    """rho = 10: two fixed-point clusters whose first feature is the settled x = +-sqrt(beta (rho - 1));
    the cluster of the lowest-index cell is -1."""
    c = CASES["fixed_points"]
    lab, f1, f2, cls = oracle(c)
    assert (cls == -1).all() and set(np.unique(lab)) == {-1, -2}
    assert np.allclose(np.abs(f1), math.sqrt(8 / 3 * 9), atol=1e-3) and (f2 == -1).all()
    assert lab[0] == -1
    assert (np.sign(f1[lab == -1]) == np.sign(f1[0])).all() and (np.sign(f1[lab == -2]) == -np.sign(f1[0])).all()


def component_rule(f1, f2, cls, eps, numb="f64"):
    """Labels by the rule the reference's host loop implies: components of the graph
    'distance <= eps' over the cells with a nonzero class; a component holding a fixed
    point (class -1) is numbered -(rank of its lowest fixed-point cell), the others
    rank of their lowest oscillating cell (class 1); components with neither and unbound
    cells stay 0."""
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import connected_components
    from scipy.spatial import cKDTree
    n = len(f1)
    t = np.float64 if numb == "f64" else np.float32
    a, b = np.asarray(f1).astype(t), np.asarray(f2).astype(t)
    act = np.asarray(cls) != 0
    fin = act & np.isfinite(a) & np.isfinite(b)
    idx = np.flatnonzero(fin)
    pairs = cKDTree(np.c_[a[idx], b[idx]].astype(np.float64)).query_pairs(float(eps) * (1 + 1e-5),
                                                                          output_type="ndarray")
    i, j = idx[pairs[:, 0]], idx[pairs[:, 1]]
    dx, dy = a[i] - a[j], b[i] - b[j]
    keep = np.sqrt(dx * dx + dy * dy) <= t(eps)
    i, j = i[keep], j[keep]
    g = coo_matrix((np.ones(len(i)), (i, j)), shape=(n, n))
    _, comp = connected_components(g, directed=False)
    cls = np.asarray(cls)
    ncomp = comp.max() + 1
    big = np.iinfo(np.int64).max
    first = {}
    for k in (-1, 1):
        cells = np.flatnonzero(act & (cls == k))
        first[k] = np.full(ncomp, big, dtype=np.int64)
        np.minimum.at(first[k], comp[cells], cells)
    comp_label = np.zeros(ncomp, dtype=np.int32)
    fp = np.flatnonzero(first[-1] < big)
    comp_label[fp[np.argsort(first[-1][fp])]] = -(np.arange(len(fp)) + 1)
    osc = np.flatnonzero((first[-1] == big) & (first[1] < big))
    comp_label[osc[np.argsort(first[1][osc])]] = np.arange(len(osc)) + 1
    return np.where(act, comp_label[comp], 0).astype(np.int32)


def synthetic(kind, n, seed, eps=0.5):
    """Features and classes of n^2 cells for one clustering case."""
    rng = np.random.default_rng(seed)
    m = n * n
    cls = rng.choice([-1, 1], size=m, p=[0.002, 0.998] if kind == "blobs" else [0.3, 0.7]).astype(np.int32)
    keep = []
    if kind == "blobs":
        centres = rng.uniform(-10, 10, size=(14, 2))
        centres[1] = centres[0] + [0.8 * eps, 0.3 * eps]  # touching pair
        which = rng.integers(0, len(centres), size=m)
        f = centres[which] + rng.normal(scale=0.15 * eps, size=(m, 2))
    elif kind == "chains":
        t = rng.uniform(0, 40, size=m)
        lane = rng.integers(0, 5, size=m)
        f = np.c_[t, lane * 1.3 * eps + rng.normal(scale=0.05 * eps, size=m)]
        f[(t > 20) & (t < 20 + 1.2 * eps), 0] += 3.0  # gaps cut the lanes
    elif kind == "heavy":
        # Two squares of about m/2 cells each whose boxes are 0.9995 eps apart along the
        # diagonal. Odd seed: A holds no cell at its box corner, so every pair is farther
        # than eps and the whole pair product is searched; even seed: one A cell sits at the
        # corner, 0.9995 eps from one B cell, and is the last A cell searched.
        half = m // 2
        q = half // 2
        jit = lambda k: rng.uniform(0.0, 0.02, size=k) * eps
        a = np.r_[np.c_[0.001 * eps + jit(q), 0.28 * eps + jit(q)],
                  np.c_[0.28 * eps + jit(half - q), 0.001 * eps + jit(half - q)]]
        s = 0.9995 / math.sqrt(2.0)
        corner = (0.3 + s) * eps
        b = np.c_[corner + jit(m - half), corner + jit(m - half)]
        b[0] = [corner, corner]
        if seed % 2 == 0:
            a[-1] = [0.3 * eps, 0.3 * eps]
        f = np.r_[a, b]
        keep = [half - 1, half]
    elif kind == "specials":
        f = rng.uniform(-3, 3, size=(m, 2))
        f[rng.random(m) < 0.3] = [1.0, 2.0]  # duplicates
        bad = rng.choice(m, size=m // 20, replace=False)
        f[bad[0::3], 0] = np.nan
        f[bad[1::3], 1] = np.inf
        f[bad[2::3], 0] = -np.inf
        cls[rng.choice(m, size=m // 25, replace=False)] = 2  # a class that never seeds
    else:
        raise ValueError(kind)
    unbound = rng.random(m) < 0.1
    unbound[keep] = False
    cls[unbound] = 0
    f[unbound] = 999.0
    return np.ascontiguousarray(f[:, 0]), np.ascontiguousarray(f[:, 1]), cls


@pytest.mark.parametrize("kind", ["blobs", "chains", "specials"])
@pytest.mark.parametrize("numb", ["f64", "f32"])
def test_component_rule_equals_literal_dbscan(kind, numb):
    f1, f2, cls = synthetic(kind, 24, seed=7)
    ref = O.dbscan_cells(f1, f2, cls, 0.5, numb)
    np.testing.assert_array_equal(component_rule(f1, f2, cls, 0.5, numb), ref)


# ------------------------------------------------------------------------------ GPU


@pytest.mark.gpu
@pytest.mark.parametrize("kind,seed", [("blobs", 1), ("chains", 2), ("heavy", 3), ("heavy", 4), ("specials", 5)])
@pytest.mark.parametrize("prec", [ucb.PREC_F64, ucb.PREC_F32])
def test_recluster_matches_oracle(kind, seed, prec):
    n = 64
    f1, f2, cls = synthetic(kind, n, seed)
    eng = ucb.Engine(0)
    lab, res = eng.run_basins_recluster("x", 3, n, 0.5, f1, f2, cls, opt=ucb.options(precision=prec))
    ref = O.dbscan_cells(f1, f2, cls, 0.5, "f64" if prec == ucb.PREC_F64 else "f32")
    np.testing.assert_array_equal(lab, ref)
    assert res.n_clusters == max(ref.max(), 0) and res.min_cluster_idx == min(ref.min(), 0)
    eng.close()


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [ucb.PREC_F64, ucb.PREC_F32])
def test_recluster_1m_cells_matches_component_rule(prec):
    n = 1024
    rng = np.random.default_rng(11)
    m = n * n
    eps = 0.01
    f = rng.uniform(0, 1, size=(m, 2)) * [12.0, 12.0]  # about 2 neighbours within eps per cell
    cls = rng.choice([-1, 1, 0], size=m, p=[0.2, 0.75, 0.05]).astype(np.int32)
    f[cls == 0] = 999.0
    eng = ucb.Engine(0)
    lab, res = eng.run_basins_recluster("x", 3, n, eps, f[:, 0].copy(), f[:, 1].copy(), cls,
                                        opt=ucb.options(precision=prec))
    ref = component_rule(f[:, 0], f[:, 1], cls, eps, "f64" if prec == ucb.PREC_F64 else "f32")
    np.testing.assert_array_equal(lab, ref)
    print(f"1M-cell clustering: {res.cluster_ms:.2f} ms, {res.n_clusters} + {-res.min_cluster_idx} clusters")
    eng.close()


# Step bodies that call a transcendental function (the forced Duffing's cos): CUDA's and
# the host's libm may round it differently in the last bit, so trajectories, and with them
# the features, agree to rounding instead of bit for bit.
TRANSCENDENTAL = {"duffing"}


def check_against_oracle(name, c, lab, f1, f2, cls, res, numb="f64"):
    rlab, rf1, rf2, rcls = oracle(c, numb)
    np.testing.assert_array_equal(cls, rcls)
    exact = name not in TRANSCENDENTAL
    for got, want, kind in ((f1, rf1, c["feature1"]), (f2, rf2, c["feature2"])):
        if not exact:
            np.testing.assert_allclose(got, want, rtol=1e-5, atol=1e-9)
        elif kind >= 6:  # log10 features: CUDA's log10 and the host's may differ in the last bit
            np.testing.assert_allclose(got, want, rtol=1e-14, atol=0)
        else:
            np.testing.assert_array_equal(got, want)
    # the clustering of the features this run produced is the reference's, label for label
    np.testing.assert_array_equal(lab, O.dbscan_cells(f1, f2, cls, c["eps_dbscan"], numb))
    if exact:
        np.testing.assert_array_equal(lab, rlab)
    # n_clusters / min_cluster_idx: the counts of oscillating / fixed-point clusters
    assert res.n_clusters == max(lab.max(), 0) and res.min_cluster_idx == min(lab.min(), 0)


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_basins_dbscan_exact_matches_oracle(name, tmp_path):
    c = dict(CASES[name], csv=str(tmp_path / "basins.csv"))
    eng = ucb.Engine(0)
    lab, f1, f2, cls, res = eng.run_basins_dbscan(request(c, precision=ucb.PREC_F64, mode=ucb.MODE_EXACT))
    check_against_oracle(name, c, lab, f1, f2, cls, res)
    n = c["n_pts"]
    grid = np.loadtxt(tmp_path / "basins.csv", delimiter=",", skiprows=2, ndmin=2)
    np.testing.assert_array_equal(grid.astype(np.int32).ravel(), lab)
    head = (tmp_path / "basins.csv").read_text().splitlines()[:2]
    assert [float(v) for v in head[0].split()] == [c["axis_x_lo"], c["axis_x_hi"]]
    assert grid.shape == (n, n)
    for suffix in ("_1.csv", "_2.csv", "_3.csv"):
        assert (tmp_path / ("basins.csv" + suffix)).exists()
    assert (tmp_path / "basins.csv_config.csv").read_text().startswith("Basins of attraction\n")
    eng.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["fixed_points", "chaotic", "unbound"])
def test_basins_dbscan_exact_f32_matches_oracle(name):
    c = CASES[name]
    eng = ucb.Engine(0)
    lab, f1, f2, cls, res = eng.run_basins_dbscan(request(c, precision=ucb.PREC_F32, mode=ucb.MODE_EXACT))
    check_against_oracle(name, c, lab, f1, f2, cls, res, "f32")
    eng.close()


@pytest.mark.gpu
def test_basins_dbscan_native_agrees():
    """The FMA-ordered step: the same fixed-point basins (the settled side agrees on >= 97 %
    of the cells; the rest sit on the basin boundary, where one rounding decides it), two
    clusters, one side each."""
    c = CASES["fixed_points"]
    eng = ucb.Engine(0)
    lab, f1, _, cls, _ = eng.run_basins_dbscan(request(c, precision=ucb.PREC_F64, mode=ucb.MODE_NATIVE))
    rlab, rf1, _, rcls = oracle(c)
    assert (cls == rcls).mean() >= 0.97
    assert (np.sign(f1) == np.sign(rf1)).mean() >= 0.97
    assert set(np.unique(lab)) == {-1, -2}
    for k in (-1, -2):  # one settled side per cluster
        assert len(np.unique(np.sign(f1[lab == k]))) == 1
    eng.close()
