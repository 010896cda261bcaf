"""The oracle (C restatement of the reference's layout pass) against the golden vectors the reference itself
produced (tests/golden/make_golden.py): bit-exact for the SGD at n_threads=1 and the t-SNE kernels."""
import numpy as np
import pytest

import sgd_cases as C
from oracle import oracle as O


def test_rng_stream_is_xorshift64star():
    # splitmix64 seeding + xorshift64* (src/rng.hpp:5-28), recomputed in Python integers
    seed = 12345
    z = (seed + 0x9E3779B97F4A7C15) & (2 ** 64 - 1)
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & (2 ** 64 - 1)
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & (2 ** 64 - 1)
    s = (z ^ (z >> 31)) | 1
    expect = []
    for _ in range(8):
        s ^= s >> 12
        s ^= (s << 25) & (2 ** 64 - 1)
        s ^= s >> 27
        expect.append((s * 0x2545F4914F6CDD1D) & (2 ** 64 - 1))
    assert [int(v) for v in O.rng_stream(seed, 8)] == expect


@pytest.mark.parametrize("case", ["default", "b1", "walk"])
def test_sgd_serial_bit_exact(golden, case):
    g = golden("sgd_small.npz")
    Y = g["Y0"].copy(); eps = g["eps"]; eons = eps.copy(); eonns = (eps / 5).astype(np.float32)
    kw = dict(a=1.7, b=0.8 if case != "b1" else 1.0, rep_a=1.7382, rep_b=1.0, seed=12345, epoch_start=0,
              epoch_end=40, alpha0=1.0, alpha1=0.0)
    if case == "default":
        kw.update(mid_pairs=g["mid_pairs"], mid_w0=0.1, mid_w1=0.0)
    if case == "walk":
        kw.update(indptr=g["indptr"], indices=g["indices"], mid_w0=0.1, mid_w1=0.0)
    O.sgd_serial(Y, g["head"], g["tail"], eps, eons, eonns, **kw)
    assert np.array_equal(Y, g[f"Y_{case}"])
    assert np.array_equal(eons, g[f"eons_{case}"]) and np.array_equal(eonns, g[f"eonns_{case}"])


@pytest.mark.parametrize("case", C.CASES)
def test_sgd_options_bit_exact(golden, ref, case):
    """InfoNCE, the gaussian / sech / tanh kernels, Adam, the norm clip, jump-graph and per-node walks, per-node b,
    the coupled repulsion kernel, exaggeration and dims 3 and 8: the oracle's serial run equals the reference's
    (stored in sgd_options.npz) bit for bit, Adam state included; and the reference run live when it is built"""
    g, opts = golden("sgd_small.npz"), golden("sgd_options.npz")
    Y, eons, eonns, kw = C.state(g, case)
    O.sgd_serial(Y, g["head"], g["tail"], g["eps"], eons, eonns, **C.oracle_kw(kw))
    Yr, eons_r, eonns_r = C.expected(g, opts, case)
    assert np.array_equal(Y, Yr)
    assert np.array_equal(eons, eons_r) and np.array_equal(eonns, eonns_r)
    if kw["optimizer"] == 1:
        for k in ("adam_m", "adam_v", "adam_t"):
            assert np.array_equal(kw[k], opts[f"{k}_{case}"])
    # every case changes the layout against the default options
    assert Y.shape != g["Y_default"].shape or not np.array_equal(Y, g["Y_default"])
    if ref is not None:
        Y2, eons2, eonns2, kw2 = C.state(g, case)
        ref.optimize_layout(Y2, g["head"], g["tail"], g["eps"], eons2, eonns2, n_threads=1, **kw2)
        assert np.array_equal(Y2, Y) and np.array_equal(eons2, eons) and np.array_equal(eonns2, eonns)


@pytest.fixture(scope="module")
def big_graph():
    return C.synthetic_graph()


@pytest.mark.parametrize("case", C.OWNER_CASES)
def test_sgd_owner_bit_exact(golden, ref, big_graph, case):
    """owner mode (parallel=1): the oracle equals the reference's run (sgd_owner.npz: Y, and sha-256 digests of
    eons, eonns and the Adam state) bit for bit, over 2 and 23 chunks, with reverse mid pairs, walks, jumps, fixed
    nodes, dims 2, 3 and 8 and distance-0 jitter draws; and the reference run live when it is built"""
    g, own = golden("sgd_small.npz"), golden("sgd_owner.npz")
    gg, Y, eons, eonns, kw, rp, rx = C.owner_state(g, case, big=big_graph)
    O.sgd_owner(Y, gg["head"], gg["tail"], gg["eps"], eons, eonns, rev_indptr=rp, rev_indices=rx, **C.oracle_kw(kw))
    assert np.array_equal(Y, own[f"Y_{case}"])
    arrays = dict(eons=eons, eonns=eonns, adam_m=kw["adam_m"], adam_v=kw["adam_v"], adam_t=kw["adam_t"])
    for entry in own[f"digests_{case}"]:
        k, h = str(entry).split(":")
        assert C.digest(arrays[k]) == h, k
    if ref is not None:
        _, Y2, eons2, eonns2, kw2, _, _ = C.owner_state(g, case, big=big_graph)
        ref.optimize_layout(Y2, gg["head"], gg["tail"], gg["eps"], eons2, eonns2, n_threads=3, parallel=1,
                            rev_indptr=rp, rev_indices=rx, **kw2)
        assert np.array_equal(Y2, Y) and np.array_equal(eons2, eons) and np.array_equal(eonns2, eonns)


def test_owner_chunks_follow_edge_quantiles(big_graph):
    """chunk boundaries at the edge quantiles, moved to node boundaries (src/layout.cpp:441-463)"""
    head = big_graph["head"]
    own, eown = O.owner_chunks(head, big_graph["Y0"].shape[0])
    E, nc = head.shape[0], own.shape[0] - 1
    assert nc == min(4096, max(1, E // 4096)) == 23
    assert own[0] == 0 and own[-1] == big_graph["Y0"].shape[0] and eown[0] == 0 and eown[-1] == E
    for t in range(1, nc):
        assert own[t] == max(head[E * t // nc], own[t - 1])
        assert eown[t] == np.searchsorted(head, own[t], "left")


def test_graph_oracle_bit_exact(golden):
    """smooth_knn and the fuzzy union restated in C equal the reference's compiled smooth_knn and its
    magnet/knn.py fuzzy_graph bit for bit (graph_small.npz): the default union, set_op_mix_ratio 0.5, and rows with
    duplicate neighbours, all-zero distances, a zero first distance and memberships that underflow to 0"""
    g = golden("graph_small.npz")
    assert np.array_equal(O.smooth_knn(g["dist"], 15), g["vals"])
    vals_e = O.smooth_knn(g["dist_e"], 15)
    assert np.array_equal(vals_e, g["vals_e"]) and (vals_e == 0).sum() > 0
    for suffix, ind, vals, mix in (("", g["ind"], g["vals"], 1.0), ("_mix", g["ind"], g["vals"], 0.5),
                                   ("_e", g["ind_e"], g["vals_e"], 1.0)):
        indptr, indices, data = O.fuzzy_union(ind, vals, None, mix)
        assert np.array_equal(indptr, g["indptr" + suffix]) and np.array_equal(indices, g["indices" + suffix])
        assert np.array_equal(data, g["data" + suffix])


def test_tsne_kernels_bit_exact(golden):
    g = golden("tsne_small.npz")
    import scipy.sparse as sp
    P = sp.csr_matrix((g["data"], g["indices"], g["indptr"]))
    Pn = P / P.sum()
    Pn = sp.csr_matrix(Pn, dtype=np.float32)
    a = O.tsne_attraction(Pn.indptr, Pn.indices, Pn.data, g["Yl"], 1.0)
    assert np.array_equal(a, g["attr"])
    assert np.array_equal(O.tsne_attraction(Pn.indptr, Pn.indices, Pn.data, g["Yl"], 0.7), g["attr07"])
    assert np.array_equal(np.array(O.bbox_2d(g["Yl"]), np.float32), g["bbox"])
    Y, U, G = g["Yl"].copy(), g["U"].copy(), g["G"].copy()
    O.tsne_step(Y, U, G, g["attr"], g["Fr"], 12.0, 1e-3, 250.0, 0.5)
    assert np.array_equal(U, g["Us"]) and np.array_equal(G, g["Gs"]) and np.array_equal(Y, g["Ys"])


def test_tsne_driver_restatement(golden):
    g = golden("tsne_small.npz")
    import scipy.sparse as sp
    P = sp.csr_matrix((g["data"], g["indices"], g["indptr"]))
    if O.reference() is None:
        pytest.skip("reference module not built")
    Y = O.optimize_tsne(P, g["Y0"].copy(), n_iter=60, early_iter=20, n_threads=1, backend="reference")
    assert np.array_equal(Y, g["Y_tsne60"])


def test_tsne_driver_variants(golden, ref):
    """the restated driver reproduces the reference's optimize_tsne bit for bit away from the defaults too (heavy
    tails, 5 interpolation points over wider boxes, late exaggeration and momentum; tsne_variants.npz)"""
    from tsne_cases import TSNE_VARIANTS
    if ref is None:
        pytest.skip("reference module not built")
    import scipy.sparse as sp
    g, v = golden("tsne_small.npz"), golden("tsne_variants.npz")
    P = sp.csr_matrix((g["data"], g["indices"], g["indptr"]))
    for name, kw in TSNE_VARIANTS.items():
        Y = O.optimize_tsne(P, g["Y0"].copy(), n_iter=60, early_iter=20, n_threads=1, backend="reference", **kw)
        assert np.array_equal(Y, v["Y_" + name]), name


@pytest.mark.parametrize("ni", [5, 3])
def test_grid_and_spectra_restatement(golden, ni):
    g = golden("fft_small.npz")
    xmin, ymin, width, nb = O.grid(g["Y"])
    assert np.allclose([xmin, ymin, width, nb], g[f"grid_{ni}"], rtol=0, atol=0)
    M, K1, K2 = O.kernel_spectra(nb, width, ni)
    assert M == int(g[f"M_{ni}"])
    assert np.array_equal([np.float64(K1).sum(), np.abs(np.float64(K1)).max()], g[f"K1h_sum_{ni}"])
    assert np.array_equal([np.float64(K2).sum(), np.abs(np.float64(K2)).max()], g[f"K2h_sum_{ni}"])


@pytest.mark.parametrize("ni", [5, 3])
def test_fft_fp64_oracle_against_reference(golden, ni):
    g = golden("fft_small.npz")
    xmin, ymin, width, nb = g[f"grid_{ni}"]
    sq, F = O.fft_repulsion_fp64(g["Y"], float(xmin), float(ymin), float(width), int(nb), ni)
    # the reference's FP32 FFT against the same interpolation with an exact convolution
    assert abs(sq - g[f"sumQ_{ni}"]) / g[f"sumQ_{ni}"] < 1e-5
    assert np.linalg.norm(F - g[f"F_{ni}"]) / np.linalg.norm(F) < 1e-4
    # and the interpolation against the exact all-pairs sums (the reference's own bounds, test_magnet.py:230-231)
    assert abs(sq - g["sumQ_exact"]) / g["sumQ_exact"] < 1e-3
    assert np.linalg.norm(F - g["F_exact"]) / np.linalg.norm(g["F_exact"]) < 2e-2


@pytest.mark.parametrize("ni", [2, 4, 7])
def test_fft_fp64_oracle_other_orders(ref, ni):
    """the FP64 restatement of the FFT pass against the reference's own FFTConv2D at interpolation orders
    other than 3 and 5 (the reference run live; it computes in FP32)"""
    if ref is None:
        pytest.skip("reference module not built")
    rng = np.random.default_rng(ni)
    Y = rng.normal(0, 8, (2500, 2)).astype(np.float32)
    xmin, ymin, width, nb = O.grid(Y)
    M, K1, K2 = O.kernel_spectra(nb, width, ni)
    conv = ref.FFTConv2D(M, ni)
    conv.set_kernels(K1, K2)
    sq_r, F_r = conv.compute(Y, xmin, ymin, width, nb, 1)
    sq, F = O.fft_repulsion_fp64(Y, xmin, ymin, width, nb, ni)
    assert abs(sq - sq_r) / abs(sq_r) < 1e-4
    assert np.linalg.norm(F - np.asarray(F_r)) / np.linalg.norm(F) < 1e-4


def test_exact_repulsion_oracle(golden):
    g = golden("fft_small.npz")
    sq, F = O.exact_repulsion(g["Y"])
    assert abs(sq - g["sumQ_exact"]) / g["sumQ_exact"] < 1e-12
    assert np.allclose(F, g["F_exact"], rtol=1e-9, atol=1e-12)


def test_schedule_record_matches_serial_run(golden):
    """the recorded draws are the ones the serial run consumes: replaying the schedule epoch by epoch advances
    eons / eonns exactly as the full run (the full run is bit-exact against the reference)"""
    g = golden("sgd_small.npz")
    eps = g["eps"]; eons = eps.copy(); eonns = (eps / 5).astype(np.float32)
    kw = dict(a=1.7, b=0.8, rep_a=1.7382, seed=12345, epoch_start=0, epoch_end=40, alpha0=1.0, alpha1=0.0,
              mid_pairs=g["mid_pairs"], mid_w0=0.1, mid_w1=0.0)
    for e in range(40):
        sampled, n_neg, off, negs, mid = O.sgd_schedule(g["Y0"].copy(), g["head"], g["tail"], eps, eons, eonns, e, **kw)
        assert negs.size == n_neg.sum()
        assert ((negs >= 0) & (negs < g["Y0"].shape[0])).all()
    assert np.array_equal(eons, g["eons_default"]) and np.array_equal(eonns, g["eonns_default"])


def test_reference_fit_and_transform_glue(ref):
    """the reference arm's served path on the compiled reference: a fit (NN-descent, fuzzy graph, schedule, mid
    pairs, SGD) and MAGNET.transform (beam-search kNN, memberships, fixed-row SGD) place new rows in their blob"""
    if ref is None:
        pytest.skip("reference module not built")
    from sklearn.neighbors import KNeighborsClassifier
    a, b = O.find_ab_params(1.0, 0.1)
    assert abs(a - 1.577) < 2e-3 and abs(b - 0.895) < 2e-3
    rng = np.random.default_rng(1)
    C = rng.normal(0, 6, (6, 16))
    y = rng.integers(0, 6, 3000)
    X = (C[y] + rng.normal(0, 1, (3000, 16))).astype(np.float32)
    Y, P = O.reference_fit(X[:2500], n_epochs=60, seed=0, a=a, b=b)
    assert Y.shape == (2500, 2) and np.isfinite(Y).all() and P.shape == (2500, 2500)
    Yn = O.reference_transform(X[:2500], P, Y, O.choose_landmarks(2500), O.transform_step(Y), X[2500:], a=a, b=b,
                               n_epochs=50, seed=1)
    assert Yn.shape == (500, 2) and np.isfinite(Yn).all()
    assert KNeighborsClassifier(10).fit(Y, y[:2500]).score(Yn, y[2500:]) > 0.9


def test_served_request_stream_is_seeded():
    """both arms of the served measurement draw the same stream: sizes in [1, 4096], Poisson gaps, fit requests
    keyed by the transform request they follow"""
    import bench as B
    rng = np.random.default_rng(0)
    C = rng.normal(0, 6, (3, 4))

    def draw(m, r):
        return (C[r.integers(0, 3, m)] + r.normal(0, 1, (m, 4))).astype(np.float32)
    s1 = B.serve_stream(draw, 40, 200.0, (50, 80), 3)
    s2 = B.serve_stream(draw, 40, 200.0, (50, 80), 3)
    assert np.array_equal(s1[0], s2[0]) and np.array_equal(s1[1], s2[1])
    assert all(np.array_equal(x, z) for x, z in zip(s1[2], s2[2]))
    assert s1[0].min() >= 1 and s1[0].max() <= 4096 and (s1[1] > 0).all()
    assert sorted(len(v) for v in s1[3].values()) == [50, 80] and all(0 < k < 40 for k in s1[3])


def test_neighbour_distance_rescale_matches_reference(golden):
    """the package's host rescale of the distance profile (power, rank exponent) equals magnet/knn.py's
    rescale_neighbor_distances bit for bit"""
    from magnet_b200.graph import rescale_neighbor_distances
    g = golden("graph_small.npz")
    assert np.array_equal(rescale_neighbor_distances(g["dist"], power=0.5, rank_exponent=0.25), g["dist_pow"])


def test_edge_schedule_matches_reference(golden):
    """the package's edge schedule (sampling frequencies, the drop rule, COO order) equals the reference's
    MAGNET._edge_schedule (magnet/__init__.py:51-66, 727-737) on the same graph bit for bit"""
    import scipy.sparse as sp
    from magnet_b200 import drivers as D
    g = golden("sgd_small.npz")
    P = sp.csr_matrix((g["data"], g["indices"], g["indptr"]))
    head, tail, eps = D.edge_schedule(P, 40)
    assert np.array_equal(head, g["head"]) and np.array_equal(tail, g["tail"]) and np.array_equal(eps, g["eps"])
    h2, t2, e2 = O.edge_schedule(P, 40)
    assert np.array_equal(h2, g["head"]) and np.array_equal(t2, g["tail"]) and np.array_equal(e2, g["eps"])


def test_find_ab_params_matches_reference(golden):
    """the package's kernel fit equals the reference's find_ab_params at six settings"""
    from magnet_b200 import drivers as D
    ab = golden("params_small.npz")["ab"]
    for kw, (a, b) in zip(C.AB_CASES, ab):
        got = D.find_ab_params(**kw)
        assert np.allclose(got, (a, b), rtol=1e-10, atol=0), (kw, got, (a, b))


@pytest.mark.parametrize("n,d,nt,seed", [(5000, 50, 1, 0), (9000, 50, 3, 11), (6000, 10, 2, 5), (3000, 17, 1, 3)])
def test_mid_near_pairs_oracle_matches_reference(ref, n, d, nt, seed):
    """the C restatement of mid_near_core (src/nndescent.cpp:731-759), the host's distance kernel, against the
    reference's compiled mid_near_pairs_dense: the same partners bit for bit"""
    if ref is None:
        pytest.skip("reference module not built")
    rng = np.random.default_rng(n + d)
    X = rng.normal(0, 3, (n, d)).astype(np.float32)
    assert np.array_equal(np.asarray(ref.mid_near_pairs_dense(X, 5, 6, seed, nt)), O.mid_near_pairs(X, 5, 6, seed, nt))


@pytest.mark.parametrize("case", ["umap10k", "components"])
def test_spectral_oracle_matches_reference(ref, case):
    """the numpy restatement of chebyshev_eigenvectors against the reference's compiled solver: the same Ritz
    vectors, column by column with the same signs"""
    if ref is None:
        pytest.skip("reference module not built")
    import os
    import scipy.sparse as sp
    from spectral_cases import inputs, three_components
    if case == "umap10k":
        g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "layout_config1.npz"))
        P = sp.csr_matrix((g["data"], g["indices"], g["indptr"]), shape=(len(g["indptr"]) - 1,) * 2)
    else:
        P = three_components()
    a = inputs(P, 2, seed=0)
    Xo = O.chebyshev_eigenvectors(*a[:3], a[3].copy(), *a[4:])
    Xr = np.asarray(ref.chebyshev_eigenvectors(*a[:3], a[3].copy(), *a[4:], -1))
    for c in range(Xo.shape[1]):
        cos = float(Xo[:, c].astype(np.float64) @ Xr[:, c]) / (np.linalg.norm(Xo[:, c]) * np.linalg.norm(Xr[:, c]))
        assert cos > 1 - 1e-6, (c, cos)
