"""Generates the golden fixtures of tests/golden/ from the reference itself (kerighan/lib-magnet 3.0.2).

Runs only where the reference checkout is available (the folder `reference` beside this repository, override with
MAGNET_REFERENCE_DIR) and its native module has been compiled by oracle/build_ref.sh. Every output is produced
by the reference's own code: its compiled `_magnet` (optimize_layout at n_threads=1 and in owner mode, FFTConv2D,
tsne_attraction, tsne_step, bbox_2d, smooth_knn) and its Python drivers (magnet/tsne.py FFTRepulsion2D /
optimize_tsne, magnet/knn.py fuzzy_graph, magnet/__init__.py edge schedule). Inputs are seeded synthetic data.

    python tests/golden/make_golden.py [sgd fft tsne sgd_options sgd_owner graph tsne_variants params]
"""
import os
import sys

import numpy as np
import scipy.sparse as sp

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("MAGNET_REFERENCE_DIR", os.path.join(os.path.dirname(ROOT), "reference"))
sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))   # the compiled reference module, importable as _magnet
sys.path.insert(0, REF)
sys.path.insert(0, HERE)

import _magnet  # noqa: E402  (the reference's native module)
from magnet import MAGNET  # noqa: E402
from magnet.knn import fuzzy_graph  # noqa: E402
from magnet.tsne import FFTRepulsion2D, optimize_tsne  # noqa: E402


def knn_graph(X, k):
    """exact kNN (self excluded) -> the reference's fuzzy graph"""
    D = ((X[:, None, :] - X[None, :, :]) ** 2).sum(-1)
    np.fill_diagonal(D, np.inf)
    ind = np.argsort(D, 1)[:, :k - 1]
    dist = np.sqrt(np.take_along_axis(D, ind, 1)).astype(np.float32)
    return fuzzy_graph(ind, dist, k)


def blobs(n, d, centers, seed, scale=5.0):
    rng = np.random.default_rng(seed)
    y = rng.integers(0, centers, n)
    C = rng.normal(0, scale, (centers, d))
    return (C[y] + rng.normal(0, 1, (n, d))).astype(np.float32), y


def sgd_fixture():
    X, y = blobs(600, 10, 5, seed=11)
    P = knn_graph(X, 15)
    n_epochs = 40
    est = MAGNET(n_epochs=n_epochs, random_state=0)
    head, tail, eps = est._edge_schedule(P, n_epochs)
    rng = np.random.default_rng(5)
    Y0 = rng.uniform(-10, 10, (600, 2)).astype(np.float32)
    mid_pairs = rng.integers(0, 600, (600, 5)).astype(np.int32)
    z = np.zeros(0, np.int32)
    out = dict(X=X, labels=y, head=head, tail=tail, eps=eps, Y0=Y0, mid_pairs=mid_pairs,
               indptr=P.indptr.astype(np.int32), indices=P.indices.astype(np.int32), data=P.data.astype(np.float32))
    cases = {
        "default": dict(b=0.8, mid=1, walk=0),
        "b1": dict(b=1.0, mid=0, walk=0),
        "walk": dict(b=0.8, mid=0, walk=1),
    }
    for name, cfg in cases.items():
        Y = Y0.copy(); eons = eps.copy(); eonns = (eps / 5).astype(np.float32)
        mp = mid_pairs if cfg["mid"] else np.zeros((0, 1), np.int32)
        mw = 0.1 if (cfg["mid"] or cfg["walk"]) else 0.0
        ip = out["indptr"] if cfg["walk"] else z
        ix = out["indices"] if cfg["walk"] else z
        _magnet.optimize_layout(Y, head, tail, eps, eons, eonns, ip, ix, 0, n_epochs, 1.0, 0.0, mw, 0.0,
                                1.7, cfg["b"], 1.7382, 1.0, 5.0, 0, 1.0, 2.0, 4, 0.25, 0, 0, 0,
                                np.zeros((0, 2), np.float32), np.zeros((0, 2), np.float32), z, 0.9, 0.999, z, mp, z, z,
                                0.0, 0, np.zeros(0, np.float32), 12345, 1, 0)
        out[f"Y_{name}"] = Y
        out[f"eons_{name}"] = eons
        out[f"eonns_{name}"] = eonns
        # the same run over 8 more seeds: the spread of the reference's own layout quality
        seeds = []
        for sd in range(1, 9):
            Y = Y0.copy(); eons = eps.copy(); eonns = (eps / 5).astype(np.float32)
            _magnet.optimize_layout(Y, head, tail, eps, eons, eonns, ip, ix, 0, n_epochs, 1.0, 0.0, mw, 0.0,
                                    1.7, cfg["b"], 1.7382, 1.0, 5.0, 0, 1.0, 2.0, 4, 0.25, 0, 0, 0,
                                    np.zeros((0, 2), np.float32), np.zeros((0, 2), np.float32), z, 0.9, 0.999, z, mp,
                                    z, z, 0.0, 0, np.zeros(0, np.float32), sd, 1, 0)
            seeds.append(Y)
        out[f"Yseeds_{name}"] = np.stack(seeds)
    np.savez_compressed(os.path.join(HERE, "sgd_small.npz"), **out)


def fft_fixture():
    out = {}
    # the reference's own test vector (tests/test_magnet.py:221-231): n = 1500, N(0, 8^2), seed 0, n_interp = 5
    rng = np.random.default_rng(0)
    Y = np.ascontiguousarray(rng.normal(0, 8, (1500, 2)).astype(np.float32))
    for ni in (5, 3):
        rep = FFTRepulsion2D(n_interp=ni, n_threads=1)
        xmin, ymin, width, nb = rep._grid(Y)
        M, K1h, K2h = rep._kernels(nb, width)
        sumQ, F = rep(Y)
        out[f"grid_{ni}"] = np.array([xmin, ymin, width, nb], np.float64)
        out[f"M_{ni}"] = np.array(M)
        # the spectra themselves are not stored (megabytes); their checksums pin oracle.kernel_spectra
        out[f"K1h_sum_{ni}"] = np.array([np.float64(K1h.real).sum(), np.abs(np.float64(K1h.real)).max()])
        out[f"K2h_sum_{ni}"] = np.array([np.float64(K2h.real).sum(), np.abs(np.float64(K2h.real)).max()])
        out[f"sumQ_{ni}"] = np.array(sumQ, np.float64)
        out[f"F_{ni}"] = F.astype(np.float32)
    D2 = ((Y[:, None, :].astype(np.float64) - Y[None, :, :]) ** 2).sum(-1)
    Q = 1.0 / (1.0 + D2)
    np.fill_diagonal(Q, 0)
    out["sumQ_exact"] = np.array(Q.sum())
    out["F_exact"] = ((Q ** 2)[:, :, None] * (Y[:, None, :].astype(np.float64) - Y[None, :, :])).sum(1)
    out["Y"] = Y
    # a t-SNE-like clustered layout (the grid's dense / sparse mix), n = 4000, n_interp = 3
    Yc, _ = blobs(4000, 2, 8, seed=3, scale=12.0)
    rep = FFTRepulsion2D(n_interp=3, n_threads=1)
    sumQ, F = rep(Yc)
    out["Yc"] = Yc
    out["sumQ_c"] = np.array(sumQ, np.float64)
    out["F_c"] = F.astype(np.float32)
    out["grid_c"] = np.array(rep._grid(Yc), np.float64)
    np.savez_compressed(os.path.join(HERE, "fft_small.npz"), **out)


def tsne_fixture():
    X, y = blobs(1200, 10, 6, seed=21)
    P = knn_graph(X, 15)
    rng = np.random.default_rng(2)
    Y0 = (rng.normal(0, 1, (1200, 2)) * 1e-4).astype(np.float32)
    Pn = sp.csr_matrix(P, dtype=np.float32)
    Pn = Pn / Pn.sum()
    ip, ix, dd = Pn.indptr.astype(np.int32), Pn.indices.astype(np.int32), Pn.data.astype(np.float32)
    Yl = (rng.normal(0, 6, (1200, 2))).astype(np.float32)
    attr = np.asarray(_magnet.tsne_attraction(ip, ix, dd, Yl, 1.0, 1))
    attr07 = np.asarray(_magnet.tsne_attraction(ip, ix, dd, Yl, 0.7, 1))
    bbox = np.array(_magnet.bbox_2d(Yl, 1), np.float32)
    U = rng.normal(0, 0.1, (1200, 2)).astype(np.float32)
    G = rng.uniform(0.5, 2.0, (1200, 2)).astype(np.float32)
    Fr = rng.normal(0, 1, (1200, 2)).astype(np.float32)
    Ys, Us, Gs = Yl.copy(), U.copy(), G.copy()
    _magnet.tsne_step(Ys, Us, Gs, attr, Fr, 12.0, 1e-3, 250.0, 0.5, 1)
    Yt = optimize_tsne(P, Y0.copy(), n_iter=60, early_iter=20, n_threads=1)
    np.savez_compressed(os.path.join(HERE, "tsne_small.npz"), X=X, labels=y,
                        indptr=P.indptr.astype(np.int32), indices=P.indices.astype(np.int32),
                        data=P.data.astype(np.float32), Y0=Y0, Yl=Yl, attr=attr, attr07=attr07, bbox=bbox,
                        U=U, G=G, Fr=Fr, Ys=Ys, Us=Us, Gs=Gs, Y_tsne60=Yt)


def sgd_options_fixture():
    """the reference's optimize_layout (n_threads=1) on each option case of sgd_cases.py: the final Y, eons, eonns
    and Adam state at seed 12345, and the 10-NN label purity of its layouts at seeds 1..8 (sgd_cases.expected reads
    them back)"""
    import sgd_cases
    g = dict(np.load(os.path.join(HERE, "sgd_small.npz")))
    out = {}
    for name in sgd_cases.CASES:
        Y, eons, eonns, kw = sgd_cases.state(g, name)
        _magnet.optimize_layout(Y, g["head"], g["tail"], g["eps"], eons, eonns, n_threads=1, **kw)
        out[f"Y_{name}"] = Y
        # the bookkeeping is stored only where it differs from the default run's (sgd_small.npz eons_default)
        if not np.array_equal(eons, g["eons_default"]):
            out[f"eons_{name}"] = eons
        if not np.array_equal(eonns, g["eonns_default"]):
            out[f"eonns_{name}"] = eonns
        if kw["optimizer"] == 1:
            out[f"adam_m_{name}"], out[f"adam_v_{name}"], out[f"adam_t_{name}"] = kw["adam_m"], kw["adam_v"], kw["adam_t"]
        pur = []
        for sd in range(1, 9):
            Y, eons, eonns, kw = sgd_cases.state(g, name, seed=sd)
            _magnet.optimize_layout(Y, g["head"], g["tail"], g["eps"], eons, eonns, n_threads=1, **kw)
            pur.append(sgd_cases.purity(Y, g["labels"]))
        out[f"purity_{name}"] = np.array(pur)
    np.savez_compressed(os.path.join(HERE, "sgd_options.npz"), **out)


def graph_fixture():
    """the reference's smooth_knn (compiled) and fuzzy_graph (magnet/knn.py) on the 600-point blobs' exact 15-NN
    (self excluded): the default union, set_op_mix_ratio 0.5, rank_exponent 0.25, and an edge case with duplicate
    neighbours, all-zero distance rows, a zero first distance and rows whose far memberships underflow to 0"""
    from magnet.knn import fuzzy_graph as ref_fuzzy_graph
    X = dict(np.load(os.path.join(HERE, "sgd_small.npz")))["X"]
    D = ((X[:, None, :].astype(np.float64) - X[None, :, :]) ** 2).sum(-1)
    np.fill_diagonal(D, np.inf)
    ind = np.argsort(D, 1, kind="stable")[:, :14].astype(np.int32)
    dist = np.sqrt(np.take_along_axis(D, ind, 1)).astype(np.float32)
    ind_e, dist_e = ind.copy(), dist.copy()
    ind_e[0:10, 5] = ind_e[0:10, 4]
    dist_e[10:20] = 0.0
    dist_e[20:30, 0] = 0.0
    dist_e[30:40, :5] = 1.0
    dist_e[30:40, 5:] = 1000.0
    out = dict(ind=ind, dist=dist, ind_e=ind_e, dist_e=dist_e)
    cases = {"": (ind, dist, {}), "_mix": (ind, dist, dict(set_op_mix_ratio=0.5)),
             "_rank": (ind, dist, dict(rank_exponent=0.25)), "_e": (ind_e, dist_e, {})}
    for suffix, (ii, dd, kw) in cases.items():
        P = ref_fuzzy_graph(ii, dd, 15, **kw)
        out["indptr" + suffix] = P.indptr.astype(np.int32)
        out["indices" + suffix] = P.indices.astype(np.int32)
        out["data" + suffix] = P.data.astype(np.float32)
    out["vals"] = np.asarray(_magnet.smooth_knn(dist, 15))
    out["vals_e"] = np.asarray(_magnet.smooth_knn(dist_e, 15))
    from magnet.knn import rescale_neighbor_distances
    out["dist_pow"] = rescale_neighbor_distances(dist, power=0.5, rank_exponent=0.25)
    np.savez_compressed(os.path.join(HERE, "graph_small.npz"), **out)


def tsne_variants_fixture():
    """the reference's optimize_tsne (magnet/tsne.py) on tsne_small.npz's graph and start, 60 iterations (20 early),
    with options other than the defaults: heavy tails (dof 0.7), 5 interpolation points per box over wider boxes,
    and late exaggeration with a higher late momentum"""
    g = dict(np.load(os.path.join(HERE, "tsne_small.npz")))
    P = sp.csr_matrix((g["data"], g["indices"], g["indptr"]))
    from tsne_cases import TSNE_VARIANTS
    out = {}
    for name, kw in TSNE_VARIANTS.items():
        out["Y_" + name] = optimize_tsne(P, g["Y0"].copy(), n_iter=60, early_iter=20, n_threads=1, **kw)
    np.savez_compressed(os.path.join(HERE, "tsne_variants.npz"), **out)


def params_fixture():
    """the reference's find_ab_params (magnet/__init__.py:26-48) at the settings of sgd_cases.AB_CASES:
    rows (a, b)"""
    from magnet import find_ab_params
    from sgd_cases import AB_CASES
    np.savez_compressed(os.path.join(HERE, "params_small.npz"),
                        ab=np.array([find_ab_params(**kw) for kw in AB_CASES], np.float64))


def sgd_owner_fixture():
    """the reference's owner mode (parallel=1, 4 threads; its result does not depend on the thread count) on each
    owner case of sgd_cases.py: the final Y and sha-256 digests of eons, eonns and the Adam state at seed 12345,
    and the 10-NN label purity of its layouts at seeds 1..8"""
    import sgd_cases
    g = dict(np.load(os.path.join(HERE, "sgd_small.npz")))
    big = sgd_cases.synthetic_graph()
    out = {}
    for name in sgd_cases.OWNER_CASES:
        for sd in [12345] + list(range(1, 9)):
            gg, Y, eons, eonns, kw, rp, rx = sgd_cases.owner_state(g, name, seed=sd, big=big)
            _magnet.optimize_layout(Y, gg["head"], gg["tail"], gg["eps"], eons, eonns, n_threads=4, parallel=1,
                                    rev_indptr=rp, rev_indices=rx, **kw)
            if sd == 12345:
                out[f"Y_{name}"] = Y
                keys = ["eons", "eonns"] + (["adam_m", "adam_v", "adam_t"] if kw["optimizer"] == 1 else [])
                arrays = dict(eons=eons, eonns=eonns, **{k: kw[k] for k in keys[2:]})
                out[f"digests_{name}"] = np.array([f"{k}:{sgd_cases.digest(arrays[k])}" for k in keys])
            else:
                out.setdefault(f"purity_{name}", []).append(sgd_cases.purity(Y, gg["labels"]))
        out[f"purity_{name}"] = np.array(out[f"purity_{name}"])
    np.savez_compressed(os.path.join(HERE, "sgd_owner.npz"), **out)


if __name__ == "__main__":
    # all fixtures, or only those named on the command line (sgd_options reads sgd_small.npz)
    todo = sys.argv[1:] or ["sgd", "fft", "tsne", "sgd_options", "sgd_owner", "graph", "tsne_variants", "params"]
    for name in todo:
        {"sgd": sgd_fixture, "fft": fft_fixture, "tsne": tsne_fixture, "sgd_options": sgd_options_fixture,
         "sgd_owner": sgd_owner_fixture, "graph": graph_fixture, "tsne_variants": tsne_variants_fixture,
         "params": params_fixture}[name]()
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))
