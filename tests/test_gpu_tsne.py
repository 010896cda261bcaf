"""t-SNE kernels and the on-device loop against the reference. Per-step forces (attraction) within 1e-5
relative per point; the step's gains and update bit-exact; the loop's layout against the reference driver's on
KL divergence (within 1 %) and neighbourhood preservation."""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def normed(g):
    P = sp.csr_matrix((g["data"], g["indices"], g["indptr"]))
    Pn = sp.csr_matrix(P / P.sum(), dtype=np.float32)
    return P, Pn


def test_attraction_per_point(mg, golden):
    g = golden("tsne_small.npz")
    _, Pn = normed(g)
    for dof, key in ((1.0, "attr"), (0.7, "attr07")):
        a = mg.tsne_attraction(Pn.indptr, Pn.indices, Pn.data, g["Yl"], dof)
        r = g[key]
        err = np.linalg.norm(a - r, axis=1)
        assert (err <= 1e-5 * np.linalg.norm(r, axis=1) + 1e-7 * np.abs(r).max()).all()


def test_attraction_any_dim(mg, golden):
    g = golden("tsne_small.npz")
    _, Pn = normed(g)
    Y5 = np.random.default_rng(1).normal(size=(Pn.shape[0], 5)).astype(np.float32)
    a = mg.tsne_attraction(Pn.indptr, Pn.indices, Pn.data, Y5, 1.0)
    r = O.tsne_attraction(Pn.indptr, Pn.indices, Pn.data, Y5, 1.0)
    assert np.allclose(a, r, rtol=1e-5, atol=1e-7 * np.abs(r).max())


def test_step_and_bbox(mg, golden):
    g = golden("tsne_small.npz")
    Y, U, G = g["Yl"].copy(), g["U"].copy(), g["G"].copy()
    mg.tsne_step(Y, U, G, g["attr"], g["Fr"], 12.0, 1e-3, 250.0, 0.5)
    assert np.array_equal(U, g["Us"]) and np.array_equal(G, g["Gs"])
    assert np.allclose(Y, g["Ys"], rtol=0, atol=1e-5)
    assert np.array_equal(np.array(mg.bbox_2d(g["Yl"]), np.float32), g["bbox"])


def kl_divergence(Pn, Y):
    """KL(P || Q) with the exact Student-t Q (dof 1) over all pairs, P normalised to sum 1"""
    Y = Y.astype(np.float64)
    D2 = ((Y[:, None, :] - Y[None, :, :]) ** 2).sum(-1)
    W = 1.0 / (1.0 + D2)
    np.fill_diagonal(W, 0.0)
    Z = W.sum()
    C = Pn.tocoo()
    p = C.data.astype(np.float64)
    q = W[C.row, C.col] / Z
    return float((p * np.log(p / q)).sum())


def knn_overlap(X, Y, k=15):
    from sklearn.neighbors import NearestNeighbors
    a = NearestNeighbors(n_neighbors=k + 1).fit(X).kneighbors(X, return_distance=False)[:, 1:]
    b = NearestNeighbors(n_neighbors=k + 1).fit(Y).kneighbors(Y, return_distance=False)[:, 1:]
    return float(np.mean([len(np.intersect1d(a[i], b[i])) / k for i in range(len(X))]))


@pytest.mark.parametrize("use_graph", [True, False])
def test_device_loop_against_reference_driver(mg, golden, use_graph):
    g = golden("tsne_small.npz")
    P, Pn = normed(g)
    Y = mg.optimize_tsne(P, g["Y0"].copy(), n_iter=60, early_iter=20, use_graph=use_graph)
    Yr = g["Y_tsne60"]
    assert np.isfinite(Y).all()
    kl, kl_r = kl_divergence(Pn, Y), kl_divergence(Pn, Yr)
    assert abs(kl - kl_r) / kl_r < 0.01
    assert abs(knn_overlap(g["X"], Y) - knn_overlap(g["X"], Yr)) < 0.02


@pytest.mark.parametrize("name", ["dof07", "interp5", "exag"])
def test_device_loop_variants_against_reference_driver(mg, golden, name):
    """the device loop away from the defaults (heavy tails, 5 interpolation points over wider boxes, late
    exaggeration and momentum) against the reference's own optimize_tsne on the same graph and start: KL within
    1 % and 15-NN overlap within 0.02"""
    from tsne_cases import TSNE_VARIANTS
    g, v = golden("tsne_small.npz"), golden("tsne_variants.npz")
    P, Pn = normed(g)
    Y = mg.optimize_tsne(P, g["Y0"].copy(), n_iter=60, early_iter=20, **TSNE_VARIANTS[name])
    Yr = v["Y_" + name]
    assert np.isfinite(Y).all()
    kl, kl_r = kl_divergence(Pn, Y), kl_divergence(Pn, Yr)
    assert abs(kl - kl_r) / kl_r < 0.01, (kl, kl_r)
    assert abs(knn_overlap(g["X"], Y) - knn_overlap(g["X"], Yr)) < 0.02


def test_device_loop_first_iteration_matches_kernels(mg, golden):
    """one iteration of the device loop equals the per-call sequence attraction -> FFT repulsion -> step"""
    g = golden("tsne_small.npz")
    P, Pn = normed(g)
    Y0 = g["Yl"].copy()
    Y1 = mg.optimize_tsne(P, Y0.copy(), n_iter=1, early_iter=1)
    rep = mg.FFTRepulsion2D(n_interp=3)
    attr = mg.tsne_attraction(Pn.indptr, Pn.indices, Pn.data, Y0, 1.0)
    sumQ, F = rep(Y0)
    Y2, U, G = Y0.copy(), np.zeros_like(Y0), np.ones_like(Y0)
    lr = max(200.0, Y0.shape[0] / 12.0)
    mg.tsne_step(Y2, U, G, attr, F, 12.0, float(1.0 / max(sumQ, 1e-12)), lr, 0.5)
    assert np.allclose(Y1, Y2, rtol=0, atol=1e-4 * np.abs(Y2).max())


def test_fft_repulsion_class_matches_reference_vector(mg, golden):
    g = golden("fft_small.npz")
    sq, F = mg.FFTRepulsion2D(n_interp=5)(g["Y"])
    assert abs(sq - g["sumQ_5"]) / g["sumQ_5"] < 1e-4
    assert np.linalg.norm(F - g["F_5"]) / np.linalg.norm(g["F_5"]) < 1e-4


def test_mid_spring(mg):
    rng = np.random.default_rng(3)
    Y = rng.normal(size=(500, 2)).astype(np.float32)
    pairs = rng.integers(0, 500, (500, 5)).astype(np.int32)
    grad = rng.normal(size=(500, 2)).astype(np.float32)
    expect = grad + 0.3 * (Y - Y[pairs].mean(1))
    mg.mid_spring(Y, pairs, grad, 0.3)
    assert np.allclose(grad, expect, rtol=1e-5, atol=1e-6)


def test_spatial_reorder_keeps_the_callers_order(mg, monkeypatch):
    """a large layout's loop sorts its points by grid box every few iterations and relabels the affinities; the
    layout comes back in the caller's order, and matches a run without the reorder to FP32 rounding (the sums run
    in another order)"""
    from magnet_b200 import graph as G
    rng = np.random.default_rng(4)
    n = 30000
    C = rng.normal(0, 6, (12, 16))
    X = (C[rng.integers(0, 12, n)] + rng.normal(0, 1, (n, 16))).astype(np.float32)
    ind, dist = G.exact_knn(X, 15)
    P = G.fuzzy_graph(ind, dist, 15)
    Y0 = (rng.normal(0, 1e-4, (n, 2))).astype(np.float32)
    monkeypatch.setenv("MAGNET_TSNE_REORDER_EVERY", "0")
    Ya = mg.optimize_tsne(P, Y0.copy(), n_iter=40, early_iter=20)
    monkeypatch.setenv("MAGNET_TSNE_REORDER_EVERY", "10")
    Yb = mg.optimize_tsne(P, Y0.copy(), n_iter=40, early_iter=20)
    assert np.isfinite(Yb).all()
    spread = float(Ya.std())
    d = np.linalg.norm(Ya - Yb, axis=1)
    assert np.median(d) < 1e-3 * spread and np.percentile(d, 99) < 1e-2 * spread, (np.median(d), spread)
    import quality   # tests/golden: the blocked FP64 KL (the whole n x n matrix would not fit at this size)
    ka, kb = quality.kl_divergence(P, Ya), quality.kl_divergence(P, Yb)
    assert abs(ka - kb) / ka < 0.002, (ka, kb)
