#!/usr/bin/env python
"""Benchmark of MAGNET's layout pass on B200: the 1M-point loss="hybrid" layout.

Workload (one "step" = one whole layout pass over it): n = 1,000,000 points in d = 50, a mixture of 100
anisotropic Gaussians (Dirichlet(1) weights, means N(0, 6^2), covariances Q diag(U[0.2, 2]) Q^T), seed 2; the
k = 15 fuzzy neighbour graph (exact kNN + UMAP smooth-kNN memberships + fuzzy union); the reference's edge
schedule for 200 epochs; 5 mid-near partners per point; a PCA initial layout rescaled as the reference rescales
its spectral init. The pass is the reference's loss="hybrid": 200 sampled SGD epochs (b = 0.6 at this n, mid
weight 0.2), recentre + rescale to std 31 sqrt(n / 70000), 300 full-batch FFT-repulsion iterations.

value: seconds per layout with every input already resident in HBM (lower is better). e2e: the same pass through
the reference-shaped numpy API (optimize_layout / optimize_tsne with host arrays in pinned memory), host-device
copies included. cpu_baseline: the reference's own CPU implementation (its compiled module, all host threads) on a
bounded sample of the same workload (SGD epochs at mid-run sampling density and full-batch iterations at the pass's
grid), extrapolated to the whole pass. --impl reference: the reference's CPU path alone, on inputs its own code
builds (NN-descent, smooth_knn and the scipy union, its mid-near partners), timing one whole pass cut into the
--steps pieces; nothing of this repository's native code is loaded in that process.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--n N]
    python bench.py --config 1|2|4 [--impl reference] [--steps K] [--warmup W]   (the other configurations)
    python bench.py --graph [--n N] [--steps K] [--warmup W] [--no-cpu-baseline]   (the fuzzy neighbour graph)

transform / transform_plain: the served form (magnet_b200.serve) on a resident 200k x 64 layout: p50 / p99
latency and points/s of transform() requests with Poisson arrivals at 200 per second, interleaved with fit
requests, on 4 slots (continuous batching) and on 1 slot (one request at a time).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "lib-magnet_b200"))

METRIC = "1M-pt layout s (mixed vs plain GPU, 15-NN ±0.005); transform p50/p99 ms"
N_EPOCHS = 200
HYBRID_ITER = 300
MID_W = 0.2


# ----------------------------------------------------------------------------------------------- workload
def make_data(n, d=50, k=100, seed=2):
    rng = np.random.default_rng(seed)
    w = rng.dirichlet(np.ones(k))
    counts = rng.multinomial(n, w)
    means = rng.normal(0, 6.0, (k, d))
    X = np.empty((n, d), np.float32)
    labels = np.empty(n, np.int32)
    s = 0
    for c in range(k):
        m = counts[c]
        Q, _ = np.linalg.qr(rng.normal(size=(d, d)))
        lam = rng.uniform(0.2, 2.0, d)
        Z = rng.standard_normal((m, d)) * np.sqrt(lam)
        X[s:s + m] = (Z @ Q.T + means[c]).astype(np.float32)
        labels[s:s + m] = c
        s += m
    perm = rng.permutation(n)
    return X[perm], labels[perm]


def find_ab(spread, min_dist, b=None):
    """the power kernel's (a, b) fitted to the (min_dist, spread) curve, b fixed when given (magnet/__init__.py:26-48);
    both arms take the pass's parameters from here"""
    from scipy.optimize import curve_fit
    xv = np.linspace(0, spread * 3, 300)
    yv = np.zeros(xv.shape)
    yv[xv < min_dist] = 1.0
    yv[xv >= min_dist] = np.exp(-(xv[xv >= min_dist] - min_dist) / spread)
    if b is None:
        params, _ = curve_fit(lambda x, a, bb: 1.0 / (1.0 + a * x ** (2 * bb)), xv, yv)
        return float(params[0]), float(params[1])
    params, _ = curve_fit(lambda x, a: 1.0 / (1.0 + a * x ** (2 * b)), xv, yv, p0=[1.0])
    return float(params[0]), float(b)


def pca_init(X, seed=2):
    """the initial layout of both arms: a 2-D PCA projection (randomised range finder) rescaled as the reference
    rescales its initial embedding (centred, max-abs 10, N(0, 1e-4) jitter; magnet/__init__.py:444-448). It stands
    in for the spectral init, which stays on the reference's host code."""
    Xc = X - X.mean(0)
    rng = np.random.default_rng(seed)
    Q, _ = np.linalg.qr(Xc @ rng.normal(size=(X.shape[1], 8)).astype(np.float32))
    for _ in range(2):
        Q, _ = np.linalg.qr(Xc @ (Xc.T @ Q))
    _, _, Vt = np.linalg.svd(Q.T @ Xc, full_matrices=False)
    Y = (Xc @ Vt[:2].T).astype(np.float32)
    Y -= Y.mean(0)
    Y *= np.float32(10.0 / max(float(np.abs(Y).max()), 1e-30))
    Y += np.random.default_rng(seed).normal(0, 1e-4, Y.shape).astype(np.float32)
    return np.ascontiguousarray(Y, dtype=np.float32)


def pass_params(n, seed=2):
    """the loss="hybrid" defaults at n points: kernel_b "size" (magnet/__init__.py:561-565), min_dist 0.05, the
    coupled repulsion exponent 1, the SGD seed drawn from random_state (:548-549)"""
    kb = float(np.clip(0.6 + 0.2 * (np.log(20000.0) - np.log(max(n, 1))) / np.log(2.0), 0.6, 0.8))
    a, b = find_ab(1.0, 0.05, kb)
    rep_a, rep_b = find_ab(1.0, 0.05, 1.0)
    return dict(a=a, b=b, rep_a=rep_a, rep_b=rep_b, seed=int(np.random.default_rng(seed).integers(0, 2 ** 62)))


def make_workload(n, seed=2):
    """the GPU arm's inputs: exact kNN, the fuzzy graph and the mid-near partners on the device (the partners are the
    reference's own for the host's thread count), the reference's edge schedule"""
    import magnet_b200 as mg
    from magnet_b200 import graph as G
    t0 = time.time()
    X, labels = make_data(n, seed=seed)
    ind, dist = G.exact_knn(X, 15)
    P = G.fuzzy_graph(ind, dist, 15)
    head, tail, eps = mg.edge_schedule(P, N_EPOCHS)
    pairs = G.mid_near_pairs(X, 5, 6, seed=seed, n_threads=-1)
    Y0 = pca_init(X, seed)
    return dict(X=X, labels=labels, P=P, head=head, tail=tail, eps=eps, pairs=pairs, Y0=Y0, n=n,
                setup_s=time.time() - t0, graph="exact kNN (device)") | pass_params(n, seed)


def make_workload_reference(n, seed=2, n_threads=-1):
    """the reference arm's inputs, from the reference's own CPU code only: its NN-descent kNN with the parameters of
    magnet/knn.py:90-122, its smooth_knn and the scipy union of magnet/knn.py:215-230, the edge schedule of
    magnet/__init__.py:727-737 and its mid-near partners (src/nndescent.cpp:731-759)"""
    from oracle import oracle as O
    R = O.reference()
    if R is None:
        raise RuntimeError("the reference module (oracle/_ref) is not built")
    t0 = time.time()
    X, labels = make_data(n, seed=seed)
    kin = min(max(14, 20), n - 1)
    n_trees = int(max(2, min(8, round(np.sqrt(n) / 40))))
    ind, d2 = R.nn_descent(X, int(kin), 50, 10, 0.001, n_trees, 30, int(seed), int(n_threads), False)
    ind = np.asarray(ind)[:, :14].astype(np.int64)
    dist = np.sqrt(np.maximum(np.asarray(d2)[:, :14], 0.0)).astype(np.float32)
    P = O.reference_fuzzy_graph(ind, dist, 15, n_threads)
    head, tail, eps = O.edge_schedule(P, N_EPOCHS)
    pairs = np.asarray(R.mid_near_pairs_dense(X, 5, 6, int(seed), int(n_threads)))
    Y0 = pca_init(X, seed)
    return dict(X=X, labels=labels, P=P, head=head, tail=tail, eps=eps, pairs=pairs, Y0=Y0, n=n,
                setup_s=time.time() - t0, graph="the reference's NN-descent") | pass_params(n, seed)


def sgd_args(w, n_epochs=N_EPOCHS, mid_w=MID_W):
    mid_len = max(1.0, 0.5 * n_epochs)
    return dict(e0=0, e1=n_epochs, alpha0=1.0, alpha1=0.0, mid0=mid_w, mid1=mid_w * max(0.0, 1.0 - n_epochs / mid_len))


# ----------------------------------------------------------------------------------------------- configs 1, 2, 4
def config1_data(n=10_000, d=50, centres=10, seed=0):
    """the loss="umap" configuration's data: ten centres N(0, 5^2 I), labels uniform, X = centre + N(0, I), from
    default_rng(seed) in that order"""
    rng = np.random.default_rng(seed)
    C = rng.normal(0, 5.0, (centres, d))
    y = rng.integers(0, centres, n)
    return (C[y] + rng.normal(0, 1, (n, d))).astype(np.float32), y


def config2_data(n=70_000, classes=10, seed=1):
    """the loss="tsne" configuration's data, image-like rows of 28 x 28 pixels: ten class prototypes, each with 149
    of the 400 pixels of the centred 20 x 20 block (about 19 % of the image) drawn U[0, 1] and the rest 0; a row is
    its class's prototype plus N(0, 0.1^2) per pixel, clipped to [0, 1]; default_rng(seed)"""
    rng = np.random.default_rng(seed)
    block = np.array([r * 28 + c for r in range(4, 24) for c in range(4, 24)])
    protos = np.zeros((classes, 784), np.float32)
    for k in range(classes):
        px = rng.choice(block, 149, replace=False)
        protos[k, px] = rng.uniform(0, 1, 149)
    y = rng.integers(0, classes, n)
    X = np.empty((n, 784), np.float32)
    for s in range(0, n, 10_000):
        e = min(n, s + 10_000)
        X[s:e] = np.clip(protos[y[s:e]] + rng.normal(0, 0.1, (e - s, 784)), 0.0, 1.0)
    return X, y


def config4_instances(count=256, d=32):
    """the batched configuration's layouts: instance i (seed 100 + i) has n = round(exp(U[ln 500, ln 20000])) points
    in d = 32 from a mixture of 3-20 Gaussians (centres N(0, 6^2 I), equal weights, unit covariance)"""
    out = []
    for i in range(count):
        rng = np.random.default_rng(100 + i)
        n = int(round(np.exp(rng.uniform(np.log(500.0), np.log(20000.0)))))
        k = int(rng.integers(3, 21))
        C = rng.normal(0, 6.0, (k, d))
        out.append((C[rng.integers(0, k, n)] + rng.normal(0, 1, (n, d))).astype(np.float32))
    return out


def perplexity_affinities(ind, d2, perplexity=30.0, n_steps=100, tol=1e-5):
    """t-SNE's input affinities, which the reference does not build (its t-SNE pass takes the fuzzy graph): per row,
    p_j|i = exp(-beta_i d2_ij) / sum_j exp(-beta_i d2_ij) over the row's neighbours (squared distances d2), with beta_i
    bisected until the row's entropy is log(perplexity) nats within tol (at most n_steps: double or halve beta until
    the target is bracketed, then halve the bracket), in FP64; then P = (P_cond + P_cond^T) / (2 n), CSR float32"""
    import scipy.sparse as sp
    d2 = np.asarray(d2, dtype=np.float64)
    n, k = d2.shape
    target = np.log(perplexity)
    beta = np.ones(n)
    lo = np.full(n, -np.inf)
    hi = np.full(n, np.inf)
    active = np.ones(n, bool)
    p = np.empty_like(d2)
    for _ in range(n_steps):
        idx = np.flatnonzero(active)
        if idx.size == 0:
            break
        e = np.exp(-d2[idx] * beta[idx, None])
        s = np.maximum(e.sum(1), 1e-8)
        H = np.log(s) + beta[idx] * (d2[idx] * e).sum(1) / s
        p[idx] = e / s[:, None]
        diff = H - target
        ok = np.abs(diff) <= tol
        active[idx[ok]] = False
        up = idx[(diff > 0) & ~ok]
        dn = idx[(diff <= 0) & ~ok]
        lo[up] = beta[up]
        beta[up] = np.where(np.isinf(hi[up]), beta[up] * 2.0, (beta[up] + hi[up]) / 2.0)
        hi[dn] = beta[dn]
        beta[dn] = np.where(np.isinf(lo[dn]), beta[dn] / 2.0, (beta[dn] + lo[dn]) / 2.0)
    rows = np.repeat(np.arange(n), k)
    C = sp.csr_matrix((p.ravel(), (rows, np.asarray(ind).ravel())), shape=(n, n))
    P = ((C + C.T) / (2.0 * n)).tocsr().astype(np.float32)
    P.eliminate_zeros()        # rows whose far neighbours' weights underflow
    P.sort_indices()
    return P


def kl_divergence(P, Y, dof=1.0, block=4096):
    """KL(P || Q) of a layout, Q the Student-t similarities normalised over all pairs i != j (FP64, blocked)"""
    import scipy.sparse as sp
    P = sp.csr_matrix(P, dtype=np.float64)
    P = P / P.sum()
    Y = np.asarray(Y, dtype=np.float64)
    n = Y.shape[0]
    Z = 0.0
    for s in range(0, n, block):
        d2 = ((Y[s:s + block, None, :] - Y[None, :, :]) ** 2).sum(-1)
        w = (1.0 + d2 / dof) ** (-dof)
        w[np.arange(w.shape[0]), np.arange(s, s + w.shape[0])] = 0.0
        Z += w.sum()
    C = P.tocoo()
    keep = C.data > 0
    q = (1.0 + ((Y[C.row[keep]] - Y[C.col[keep]]) ** 2).sum(-1) / dof) ** (-dof) / Z
    return float((C.data[keep] * np.log(C.data[keep] / q)).sum())


def exact_knn_cpu(X, k):
    """(indices (n, k), squared distances (n, k)) of the k nearest other rows, exact, on the host's cores"""
    from sklearn.neighbors import NearestNeighbors
    d, i = NearestNeighbors(n_neighbors=k + 1, algorithm="brute", n_jobs=-1).fit(X).kneighbors(X)
    return i[:, 1:].astype(np.int64), (d[:, 1:].astype(np.float64) ** 2)


def config_leg(cfg, impl, steps, warmup):
    """one JSON line for configuration 1 (10k umap SGD, 500 epochs, n_threads = 1) or 2 (70k tsne, perplexity 30,
    750 iterations with 250 of early exaggeration 12): the layout pass's seconds per layout with device-resident
    inputs (for configuration 1 the counter mode, with the serial stream mode, the reference's single stream, beside
    it), or the reference's CPU path (impl "reference"), with 15-NN preservation and KL of the result"""
    nt = os.cpu_count() or 1
    if cfg == 1:
        import scipy.sparse as sp
        g = dict(np.load(os.path.join(ROOT, "tests", "golden", "layout_config1.npz")))
        X, _ = config1_data()
        P = sp.csr_matrix((g["data"], g["indices"], g["indptr"]), shape=(X.shape[0],) * 2)
        n_epochs, seed = int(g["n_epochs"]), int(g["seed"])
        config = {"workload": "umap layout, n=10000, d=50, 10 Gaussians, seed 0, k=15 (the reference's NN-descent "
                              "graph and spectral init, captured from its fit), 500 epochs, n_threads=1",
                  "n_points": 10000, "l2": "inputs in L2 (6 MB of edges); no flush between epochs, as in a layout pass"}
        out = {"metric": "10k umap layout s (500 epochs, n_threads=1)", "unit": "s", "steps": steps,
               "warmup": warmup, "higher_is_better": False, "dtype": "f32", "data": "synthetic", "config": config}
        if impl == "reference":
            from oracle import oracle as O
            head, tail, eps = O.edge_schedule(P, n_epochs)
            times, Y = [], None
            for i in range(warmup + steps):
                Y = g["Y0"].copy()
                t0 = time.perf_counter()
                O.optimize_sgd(Y, head, tail, eps, n_epochs, mid_weight=float(g["mid_w"]), mid_pairs=g["mid_pairs"],
                               backend="reference", n_threads=1, seed=seed, a=float(g["a"]), b=float(g["b"]),
                               rep_a=float(g["rep_a"]), rep_b=float(g["rep_b"]), indptr=P.indptr, indices=P.indices)
                if i >= warmup:
                    times.append(time.perf_counter() - t0)
            out |= {"impl": "reference", "cores": 1, "value": round(statistics.median(times), 4),
                    "knn15": round(knn_preservation(X, Y), 4), "kl": round(kl_divergence(P, Y), 4)}
        else:
            import torch
            import magnet_b200 as mg
            head, tail, eps = mg.edge_schedule(P, n_epochs)
            dev = torch.device("cuda", torch.cuda.current_device())
            t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
            hd, td, ed, pd = t(head), t(tail), t(eps), t(g["mid_pairs"])
            ipd, ixd = t(P.indptr.astype(np.int32)), t(P.indices.astype(np.int32))
            Y0 = t(g["Y0"])
            eonns0 = (ed / 5.0).contiguous()
            z, zf = torch.zeros(0, dtype=torch.int32, device=dev), torch.zeros(0, dtype=torch.float32, device=dev)
            z2 = torch.zeros((0, 2), dtype=torch.float32, device=dev)

            def run(mode):
                # MAGNET._optimize's one call over [0, 500): alpha 1 -> 0, mid weight mid_w -> 0 (its window is 250
                # epochs, so it reaches 0 at the end of the call)
                Y, eons, eonns = Y0.clone(), ed.clone(), eonns0.clone()
                mg.optimize_layout(Y, hd, td, ed, eons, eonns, ipd, ixd, 0, n_epochs, 1.0, 0.0, float(g["mid_w"]), 0.0,
                                   float(g["a"]), float(g["b"]), float(g["rep_a"]), float(g["rep_b"]), 5.0, 0, 1.0,
                                   2.0, 4, 0.25, 0, 0, 0, z2, z2, z, 0.9, 0.999, z, pd, z, z, 0.0, 0, zf, seed, -1, 0,
                                   None, None, 1 if mode == "serial" else 0)
                return Y
            for mode in ("serial", "hogwild"):
                for _ in range(warmup):
                    run(mode)
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                for _ in range(steps):
                    Y = run(mode)
                e1.record()
                torch.cuda.synchronize()
                Yh = Y.cpu().numpy()
                out[mode] = {"value": round(e0.elapsed_time(e1) / steps / 1000, 4),
                             "knn15": round(knn_preservation(X, Yh), 4), "kl": round(kl_divergence(P, Yh), 4)}
            # the value is the device's own mode (hogwild counter draws); the serial stream mode, which replays the
            # reference's single stream on one device thread, is a parity mode and is reported beside it
            out |= {"value": out["hogwild"]["value"], "knn15": out["hogwild"]["knn15"], "kl": out["hogwild"]["kl"]}
        print(json.dumps(out))
        return
    # configuration 2
    X, _ = config2_data()
    n = X.shape[0]
    t0 = time.time()
    if impl == "reference":
        ind, d2 = exact_knn_cpu(X, 90)
    else:
        from magnet_b200 import graph as G
        ind, dist = G.exact_knn(X, 91)
        d2 = dist.astype(np.float64) ** 2
    P = perplexity_affinities(ind, d2, 30.0)
    Y0 = pca_init(X, 1)
    Y0 = np.ascontiguousarray(Y0 / max(float(Y0[:, 0].std()), 1e-12) * 1e-4, dtype=np.float32)
    setup_s = time.time() - t0
    config = {"workload": "tsne layout, n=70000, d=784 image-like rows (10 prototypes), seed 1, perplexity 30 "
                          "(90 neighbours), 750 iterations with 250 of early exaggeration 12, 3 points per box",
              "n_points": n, "l2": "inputs larger than L2 for the affinities (%d MB)" % (P.nnz * 8 // 2 ** 20)}
    if impl == "reference":
        from oracle import oracle as O
        for _ in range(warmup):
            O.TsneRun(P, Y0.copy(), n_iter=1, early_iter=1, n_threads=-1, backend="reference").advance(1)
        run = O.TsneRun(P, Y0.copy(), n_iter=750, early_iter=250, n_threads=-1, backend="reference")
        times = []
        for k in split_iterations(750, steps):
            t1 = time.perf_counter()
            run.advance(k)
            times.append(time.perf_counter() - t1)
        Y = run.Y
        line = {"impl": "reference", "cores": nt, "value": round(sum(times), 3),
                "sample": "the whole 750 iterations timed in %d consecutive pieces" % steps}
    else:
        import torch
        import magnet_b200 as mg
        dev = torch.device("cuda", torch.cuda.current_device())
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        Pn = P / P.sum()
        ipd, ixd, dd = t(Pn.indptr.astype(np.int32)), t(Pn.indices.astype(np.int32)), t(Pn.data.astype(np.float32))
        Yd0 = t(Y0)
        Yd = torch.empty_like(Yd0)

        def run():
            Yd.copy_(Yd0)
            mg._native.optimize_tsne(ipd, ixd, dd, Yd, 750, 250, 12.0, 1.0, -1.0, 0.5, 0.8, 3, 0.7, 1.0, 20, 1000, 0,
                                     True)
        for _ in range(warmup):
            run()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            run()
        e1.record()
        torch.cuda.synchronize()
        Y = Yd.cpu().numpy()
        line = {"value": round(e0.elapsed_time(e1) / steps / 1000, 4)}
    out = {"metric": "70k tsne layout s (750 iterations)", "unit": "s", "steps": steps, "warmup": warmup,
           "higher_is_better": False, "dtype": "f32", "data": "synthetic", "config": config,
           "inputs": {"knn": "exact, on the host's cores" if impl == "reference" else "exact, on the device",
                      "nnz": int(P.nnz), "setup_s": round(setup_s, 1)},
           "knn15": round(knn_preservation(X, Y), 4), "kl": round(kl_divergence(P, Y), 4)} | line
    print(json.dumps(out))


def config4_leg(impl, steps, warmup, count=256, n_iter=500):
    """the batched form: `count` independent perplexity-30 t-SNE layouts of 500-20,000 points, 500 iterations each
    (166 of early exaggeration 12, MAGNET's default min(250, n_iter // 3) for loss="tsne"); layouts/s of the batch
    (one CUDA graph per iteration, the layouts as branches, launch shapes from the autotuner) beside the plain device
    form (one optimize_tsne call per layout, in sequence), or the reference's loop of optimize_tsne calls on the
    host's cores over a size-stratified sample of the layouts (impl "reference"); per-layout KL and 15-NN on the
    sample"""
    Xs = config4_instances(count)
    early = min(250, n_iter // 3)
    sample = sorted(range(count), key=lambda i: Xs[i].shape[0])[::16]
    t0 = time.time()
    Ps, Y0s = [], []
    for i, X in enumerate(Xs):
        if impl == "reference":
            ind, d2 = exact_knn_cpu(X, 90)
        else:
            from magnet_b200 import graph as G
            ind, dist = G.exact_knn(X, 91)
            d2 = dist.astype(np.float64) ** 2
        Ps.append(perplexity_affinities(ind, d2, 30.0))
        Y0 = pca_init(X, 100 + i)
        Y0s.append(np.ascontiguousarray(Y0 / max(float(Y0[:, 0].std()), 1e-12) * 1e-4, dtype=np.float32))
    setup_s = time.time() - t0
    config = {"workload": "%d t-SNE layouts, n log-uniform in [500, 20000] (total %d), d=32, 3-20 Gaussians each, "
                          "seeds 100-%d, perplexity 30, %d iterations (%d early)" % (count, sum(len(X) for X in Xs),
                                                                                    99 + count, n_iter, early),
              "n_layouts": count}

    def quality_of(Ys):
        return {"kl": [round(kl_divergence(Ps[i], Ys[i]), 4) for i in sample],
                "knn15": [round(knn_preservation(Xs[i], Ys[i]), 4) for i in sample]}
    if impl == "reference":
        from oracle import oracle as O
        times, Ys = [], {}
        for i in sample:
            t1 = time.perf_counter()
            Ys[i] = O.optimize_tsne(Ps[i], Y0s[i].copy(), n_iter=n_iter, early_iter=early, n_threads=-1,
                                    backend="reference")
            times.append(time.perf_counter() - t1)
        out = {"impl": "reference", "value": round(len(sample) / sum(times), 4), "cores": os.cpu_count(),
               "sample": "%d of the %d layouts (every 16th by size), each a whole optimize_tsne pass" % (len(sample),
                                                                                                        count),
               "per_layout_s": [round(t, 3) for t in times], "quality": quality_of(Ys)}
    else:
        import torch
        import magnet_b200 as mg
        from magnet_b200 import autotune as A
        Ys = [Y.copy() for Y in Y0s]
        mg.optimize_tsne_batch(Ps, Ys, n_iter=n_iter, early_iter=early)     # tunes once for this shape (cached)
        key = A.batch_key([len(X) for X in Xs], [P.nnz for P in Ps])
        choice = A.lookup(key) or {}
        graphs = [(P.indptr.astype(np.int32), P.indices.astype(np.int32), P.data.astype(np.float32)) for P in Ps]
        batch = mg._native.TsneBatch(graphs, n_iter=n_iter, early_iter=early,
                                     threads_per_row=int(choice.get("threads_per_row", 0)),
                                     branches=int(choice.get("branches", 32)))
        dev = torch.device("cuda", torch.cuda.current_device())
        Yd0 = [torch.from_numpy(Y).to(dev) for Y in Y0s]
        Yd = [torch.empty_like(Y) for Y in Yd0]
        for _ in range(warmup):
            for a, b in zip(Yd, Yd0):
                a.copy_(b)
            batch.run(Yd)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        for _ in range(steps):
            for a, b in zip(Yd, Yd0):
                a.copy_(b)
            batch.run(Yd)
        torch.cuda.synchronize()
        batched_s = (time.perf_counter() - t1) / steps
        Yb = [Y.cpu().numpy() for Y in Yd]
        t1 = time.perf_counter()
        for a, b, G_ in zip(Yd, Yd0, graphs):
            a.copy_(b)
            mg._native.optimize_tsne(G_[0], G_[1], G_[2], a, n_iter, early, 12.0, 1.0, -1.0, 0.5, 0.8, 3, 0.7, 1.0,
                                     20, 1000, int(choice.get("threads_per_row", 0)), True)
        torch.cuda.synchronize()
        plain_s = time.perf_counter() - t1
        out = {"value": round(count / batched_s, 3), "batched_s": round(batched_s, 3),
               "plain": {"value": round(count / plain_s, 3), "s": round(plain_s, 3)},
               "speedup_vs_plain": round(plain_s / batched_s, 2), "autotune": choice,
               "kernels_per_iteration": int(batch.kernels_per_iteration), "quality": quality_of(Yb)}
    line = {"metric": "batched t-SNE layouts/s (256 layouts, 500 iterations)", "unit": "layouts/s",
            "higher_is_better": True, "steps": steps, "warmup": warmup, "dtype": "f32", "data": "synthetic",
            "config": config, "inputs": {"setup_s": round(setup_s, 1), "sample": sample}} | out
    print(json.dumps(line))


# ----------------------------------------------------------------------------------------------- GPU arm
class GpuPass:
    """the hybrid pass on device-resident inputs (value) or through host arrays (e2e)"""

    def __init__(self, w):
        import torch
        import magnet_b200 as mg
        self.mg, self.torch, self.w = mg, torch, w
        dev = torch.device("cuda", torch.cuda.current_device())
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        P = w["P"]
        self.d = dict(head=t(w["head"]), tail=t(w["tail"]), eps=t(w["eps"]), pairs=t(w["pairs"]), Y0=t(w["Y0"]),
                      indptr=t(P.indptr.astype(np.int32)), indices=t(P.indices.astype(np.int32)),
                      data=t(P.data.astype(np.float32)))
        self.d["eonns0"] = (self.d["eps"] / 5.0).contiguous()
        self.Y = torch.empty_like(self.d["Y0"])
        self.eons = torch.empty_like(self.d["eps"])
        self.eonns = torch.empty_like(self.d["eps"])
        self.z = torch.zeros(0, dtype=torch.int32, device=dev)
        self.zf = torch.zeros(0, dtype=torch.float32, device=dev)
        self.z2 = torch.zeros((0, 2), dtype=torch.float32, device=dev)
        # pinned host copies for the end-to-end pass
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
        self.h = dict(head=pin(w["head"]), tail=pin(w["tail"]), eps=pin(w["eps"]), pairs=pin(w["pairs"]),
                      indptr=pin(P.indptr.astype(np.int32)), indices=pin(P.indices.astype(np.int32)),
                      data=pin(P.data.astype(np.float32)), Y0=pin(w["Y0"]))
        self.hY = pin(w["Y0"])
        self.heons = pin(w["eps"])
        self.heonns = pin((w["eps"] / 5.0).astype(np.float32))
        self.target = 31.0 * np.sqrt(w["n"] / 70000.0)

    def _sgd(self, Y, head, tail, eps, eons, eonns, pairs, z, zf, z2, n_epochs=N_EPOCHS):
        w, s = self.w, sgd_args(self.w, n_epochs)
        self.mg.optimize_layout(Y, head, tail, eps, eons, eonns, z, z, s["e0"], s["e1"], s["alpha0"], s["alpha1"],
                                s["mid0"], s["mid1"], w["a"], w["b"], w["rep_a"], w["rep_b"], 5.0, 0, 1.0, 2.0, 4,
                                0.25, 0, 0, 0, z2, z2, z, 0.9, 0.999, z, pairs, z, z, 0.0, 0, zf, w["seed"], -1, 0,
                                None, None, 0)

    def step_device(self):
        d = self.d
        self.Y.copy_(d["Y0"]); self.eons.copy_(d["eps"]); self.eonns.copy_(d["eonns0"])
        self._sgd(self.Y, d["head"], d["tail"], d["eps"], self.eons, self.eonns, d["pairs"], self.z, self.zf, self.z2)
        self.mg.center_scale(self.Y, float(self.target))
        self.mg._native.optimize_tsne(d["indptr"], d["indices"], d["data"], self.Y, HYBRID_ITER, 0, 12.0, 1.0, -1.0,
                                      0.5, 0.8, 3, 0.7, 1.0, 20, 1000, 0, True)

    def step_e2e(self):
        """the reference-facing call sequence with host (pinned) arrays; returns (h2d, d2h) bytes"""
        h = self.h
        np.copyto(self.hY, h["Y0"]); np.copyto(self.heons, h["eps"]); np.copyto(self.heonns, h["eps"] / np.float32(5.0))
        z = np.zeros(0, np.int32); zf = np.zeros(0, np.float32); z2 = np.zeros((0, 2), np.float32)
        self._sgd(self.hY, h["head"], h["tail"], h["eps"], self.heons, self.heonns, h["pairs"], z, zf, z2)
        Y = self.hY
        Y -= Y.mean(0)
        Y *= np.float32(self.target / max(float(Y[:, 0].std()), 1e-12))
        self.mg._native.optimize_tsne(h["indptr"], h["indices"], h["data"], Y, HYBRID_ITER, 0, 12.0, 1.0, -1.0,
                                      0.5, 0.8, 3, 0.7, 1.0, 20, 1000, 0, True)
        nb = lambda *a: sum(int(x.nbytes) for x in a)
        h2d = nb(self.hY, h["head"], h["tail"], h["eps"], self.heons, self.heonns, h["pairs"]) + \
            nb(h["indptr"], h["indices"], h["data"], self.hY)
        d2h = nb(self.hY, self.heons, self.heonns) + nb(self.hY)
        return h2d, d2h

    def result(self):
        return self.Y.cpu().numpy()


# ----------------------------------------------------------------------------------------------- reference CPU path
def reference_sgd(R, w, Y, eons, eonns, e0, e1, n_threads):
    """one optimize_layout call of the reference over epochs [e0, e1) with the pass's linear schedules (as
    MAGNET._optimize makes them, magnet/__init__.py:796-839)"""
    z = np.zeros(0, np.int32)
    alpha = lambda e: 1.0 - e / N_EPOCHS
    mid = lambda e: MID_W * (1.0 - e / N_EPOCHS)   # the single call's linear interpolation of sgd_args
    R.optimize_layout(Y, w["head"], w["tail"], w["eps"], eons, eonns, z, z, e0, e1, alpha(e0), alpha(e1), mid(e0),
                      mid(e1), w["a"], w["b"], w["rep_a"], w["rep_b"], 5.0, 0, 1.0, 2.0, 4, 0.25, 0, 0, 0,
                      np.zeros((0, 2), np.float32), np.zeros((0, 2), np.float32), z, 0.9, 0.999, z, w["pairs"], z, z,
                      0.0, 0, np.zeros(0, np.float32), w["seed"], n_threads, 0)


def rescale(Y, n):
    """the hybrid pass's recentre + rescale to std 31 sqrt(n / 70000) (magnet/__init__.py:695-696)"""
    Y -= Y.mean(0)
    Y *= np.float32(31.0 * np.sqrt(n / 70000.0) / max(float(Y[:, 0].std()), 1e-12))
    return Y


def split_iterations(total, pieces):
    """total iterations in `pieces` near-equal consecutive runs"""
    return [total // pieces + (1 if j < total % pieces else 0) for j in range(pieces)] if pieces > 0 else []


class ReferencePass:
    """The whole hybrid pass on the reference's CPU path (its compiled module on all host threads, driven as
    MAGNET.fit drives it for loss="hybrid", magnet/__init__.py:683-700), cut into `pieces` consecutive timed
    pieces: piece 0 is the SGD pass (one optimize_layout call of 200 epochs, as the reference makes it) and the
    rescale, pieces 1.. are the 300 full-batch iterations in near-equal runs of the reference's t-SNE loop
    (magnet/tsne.py:132-184, the loop restated in oracle.TsneRun, state carried from piece to piece). The pieces
    together run one whole pass; their times add up to the seconds per layout."""

    def __init__(self, w, pieces, n_threads):
        from oracle import oracle as O
        self.O, self.R, self.w, self.nt = O, O.reference(), w, n_threads
        self.pieces = max(1, int(pieces))
        self.iters = split_iterations(HYBRID_ITER, self.pieces - 1)
        self.Y = self.run = None

    def piece(self, j):
        w = self.w
        if j == 0:
            self.Y = w["Y0"].copy()
            eons, eonns = w["eps"].copy(), (w["eps"] / np.float32(5.0)).astype(np.float32)
            reference_sgd(self.R, w, self.Y, eons, eonns, 0, N_EPOCHS, self.nt)
            rescale(self.Y, w["n"])
            self.run = self.O.TsneRun(w["P"], self.Y, n_iter=HYBRID_ITER, early_iter=0, exaggeration=1.0,
                                      n_threads=self.nt, backend="reference")
            if self.pieces == 1:
                self.run.advance(HYBRID_ITER)
        else:
            self.run.advance(self.iters[j - 1])
        return self.run.Y

    def warmup(self):
        """one SGD epoch and one iteration on copies (pages in the inputs and the module)"""
        w = self.w
        Y = w["Y0"].copy()
        reference_sgd(self.R, w, Y, w["eps"].copy(), (w["eps"] / np.float32(5.0)).astype(np.float32), 0, 1, self.nt)
        self.O.TsneRun(w["P"], rescale(Y, w["n"]), n_iter=1, early_iter=0, n_threads=self.nt,
                       backend="reference").advance(1)


def reference_sample(w, Y_tsne=None, sgd_epochs=2, tsne_iters=2):
    """The reference's CPU implementation (its compiled module, all host threads) on a bounded sample: SGD epochs
    at mid-run sampling density and full-batch iterations of the hybrid pass; returns seconds per whole layout
    (extrapolated) and the sample's details. The per-epoch and per-iteration costs are the difference between a
    run of 1 + k units and a run of 1 unit, so that the one-time set-up of a call (argument checks, the kernel
    spectra of a new grid) is not counted; a whole pass pays it once per call segment or grid change."""
    from oracle import oracle as O
    R = O.reference()
    if R is None:
        raise RuntimeError("the reference module (oracle/_ref) is not built")
    nt = os.cpu_count() or 1
    n = w["n"]
    rng = np.random.default_rng(5)
    eps = w["eps"]
    e_mid = N_EPOCHS // 2
    eons0 = (e_mid + rng.uniform(0, 1, eps.size).astype(np.float32) * eps).astype(np.float32)
    eonns0 = (eons0 - eps / 5.0).astype(np.float32)

    def sgd(k):
        Y, eons, eonns = w["Y0"].copy(), eons0.copy(), eonns0.copy()
        t0 = time.perf_counter()
        reference_sgd(R, w, Y, eons, eonns, e_mid, e_mid + k, nt)
        return time.perf_counter() - t0

    if Y_tsne is None:
        Y_tsne = rescale(w["Y0"].copy(), n)

    def tsne(k):
        t0 = time.perf_counter()
        O.optimize_tsne(w["P"], Y_tsne.copy(), n_iter=k, early_iter=0, exaggeration=1.0, n_threads=nt,
                        backend="reference")
        return time.perf_counter() - t0

    t_sgd = max(sgd(1 + sgd_epochs) - sgd(1), 0.0) / sgd_epochs
    t_it = max(tsne(1 + tsne_iters) - tsne(1), 0.0) / tsne_iters
    total = t_sgd * N_EPOCHS + t_it * HYBRID_ITER
    sample = (f"{sgd_epochs} SGD epochs (mid-run schedule density) at {t_sgd:.3f} s/epoch and {tsne_iters} "
              f"full-batch iterations at {t_it:.3f} s/iteration on the {n}-point workload (each the difference of "
              f"a run of 1 + k units and of 1 unit, so a call's one-time set-up is not counted), extrapolated to "
              f"{N_EPOCHS} epochs + {HYBRID_ITER} iterations")
    return total, nt, sample


# ----------------------------------------------------------------------------------------------- measurement helpers
class Clocks:
    def __init__(self, index):
        self.f = None
        self.p = None
        self.index = index

    def __enter__(self):
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                text=True)
        except (OSError, FileNotFoundError):
            self.p = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.p is not None:
            self.p.terminate()
            try:
                self.out, _ = self.p.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()
                self.out, _ = self.p.communicate()

    def summary(self):
        rows = []
        for line in (self.out or "").strip().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 7:
                try:
                    rows.append((float(parts[0]), float(parts[1]), parts[3:7]))
                except ValueError:
                    pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        active = sorted({names[i] for r in rows for i, v in enumerate(r[2]) if v.lower().startswith("active")})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": active, "samples": len(rows)}


def knn_preservation(X, Y, k=15, n_query=5000, seed=0):
    """15-NN preservation of benchmarks/metrics.py:52-62: the exact k-NN of a seeded 5,000-row query subsample in
    the data and in the layout, mean overlap / k. Computed on the host's cores (brute force in the data, a k-d tree
    in the layout) with the same code in both arms, so the two figures compare like with like."""
    from sklearn.neighbors import NearestNeighbors
    from scipy.spatial import cKDTree
    rng = np.random.default_rng(seed)
    q = np.sort(rng.choice(X.shape[0], min(n_query, X.shape[0]), replace=False))
    hi = NearestNeighbors(n_neighbors=k + 1, algorithm="brute", n_jobs=-1).fit(X).kneighbors(
        X[q], return_distance=False)
    Yd = np.asarray(Y, dtype=np.float64)
    lo = cKDTree(Yd).query(Yd[q], k + 1, workers=-1)[1]

    def drop_self(rows):
        return [[j for j in r if j != i][:k] for i, r in zip(q, rows)]
    a, b = drop_self(hi), drop_self(lo)
    return float(np.mean([len(np.intersect1d(a[i], b[i])) / k for i in range(len(q))]))


def precision_study(Y, n_sub=10_000, seed=0):
    """the FFT pass's error on a 10k-point subsample of a layout: the device's FP32 spread / FFT / gather with the
    FP64 Z reduction (FFTRepulsion2D, the reference's grid rule) against the direct FP64 all-pairs sums of the same
    points (sumQ = sum_{i != j} (1 + |y_i - y_j|^2)^-1, F_i = sum_j (1 + |y_i - y_j|^2)^-2 (y_i - y_j)), computed
    in FP64 on the device"""
    import torch
    import magnet_b200 as mg
    rng = np.random.default_rng(seed)
    Ys = np.ascontiguousarray(Y[rng.choice(Y.shape[0], min(n_sub, Y.shape[0]), replace=False)], dtype=np.float32)
    sq, F = mg.FFTRepulsion2D(n_interp=3)(Ys)
    Yd = torch.from_numpy(Ys.astype(np.float64)).cuda()
    s64 = torch.zeros((), dtype=torch.float64, device="cuda")
    F64 = torch.zeros_like(Yd)
    for a in range(0, Yd.shape[0], 2048):
        diff = Yd[a:a + 2048, None, :] - Yd[None, :, :]
        q = 1.0 / (1.0 + (diff * diff).sum(-1))
        idx = torch.arange(a, min(a + 2048, Yd.shape[0]), device="cuda")
        q[idx - a, idx] = 0.0
        s64 += q.sum()
        F64[a:a + 2048] = ((q * q)[:, :, None] * diff).sum(1)
    s64 = float(s64)
    F64 = F64.cpu().numpy()
    F = np.asarray(F, dtype=np.float64)
    return {"n": int(Ys.shape[0]), "sumQ_rel_err": float(abs(sq - s64) / s64),
            "F_rel_rms_err": float(np.linalg.norm(F - F64) / np.linalg.norm(F64)),
            "F_max_rel_err": float(np.abs(F - F64).max() / np.abs(F64).max()),
            "against": "direct FP64 all-pairs sums on the device"}


def roofline(w, gp, peak):
    """per-stage CUDA-event times of the t-SNE iteration and of the SGD epoch kernel, the dominant kernel's
    achieved GB/s against its algorithmic bytes"""
    import torch
    peaks, peak_src = peak
    mg = gp.mg
    d = gp.d
    n = w["n"]
    # SGD epochs: one kernel per epoch (plus the row-pointer set-up of the call)
    gp.Y.copy_(d["Y0"]); gp.eons.copy_(d["eps"]); gp.eonns.copy_(d["eonns0"])
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    gp._sgd(gp.Y, d["head"], d["tail"], d["eps"], gp.eons, gp.eonns, d["pairs"], gp.z, gp.zf, gp.z2)
    e1.record(st)
    torch.cuda.synchronize()
    sgd_ms = e0.elapsed_time(e1) / N_EPOCHS
    mg.center_scale(gp.Y, float(gp.target))
    n_prof = 30
    prof = mg._native.optimize_tsne_profiled(d["indptr"], d["indices"], d["data"], gp.Y, n_prof, 0, 12.0, 1.0, -1.0,
                                             3, 0.7, 1.0)
    nb_, N, M, Mh = prof["grid"]
    E = int(w["head"].size)
    S = float(np.floor((N_EPOCHS - 1) / w["eps"].astype(np.float64)).sum()) / N_EPOCHS   # samples per epoch
    nnz = int(w["P"].nnz)
    stages = {k: prof[k] / n_prof for k in ("bbox_grid", "twiddles", "spectra", "spread", "row_fwd", "col_conv",
                                             "row_inv", "gather_attr_step")}
    # algorithmic bytes per launch (each array element counted once per use)
    alg = {
        "sgd_epoch": 4 * E + 101 * S,
        "col_conv": 48.0 * N * Mh + 8.0 * M * Mh,
        "row_fwd": 12.0 * N * N + 24.0 * N * Mh,
        "row_inv": 24.0 * N * Mh + 12.0 * N * N,
        "spread": 8.0 * n + 12.0 * N * N,
        "gather_attr_step": 12.0 * N * N + 8.0 * n + 16.0 * nnz + 4.0 * n + 64.0 * n,
        "spectra": 2 * (8.0 * M * (M // 2 + 1) + 8.0 * Mh * (M // 2 + 1)) + 8.0 * M * Mh,
    }
    share = {"sgd_epoch": sgd_ms * N_EPOCHS}
    for k, v in stages.items():
        share[k] = v * HYBRID_ITER
    dom = max((k for k in share if k in alg), key=lambda k: share[k])
    ms = sgd_ms if dom == "sgd_epoch" else stages[dom]
    achieved = alg[dom] / (ms * 1e-3) / 1e9
    traffic = measured_traffic(dom, n)
    # the FFT pass is the four stages from the spread to the potentials (the gather is timed with the iteration)
    fft_pass_bytes = alg["spread"] + alg["row_fwd"] + alg["col_conv"] + alg["row_inv"]
    fft_pass_ms = stages["spread"] + stages["row_fwd"] + stages["col_conv"] + stages["row_inv"]
    return {
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peaks,
                     "unit": "GB/s", "frac": round(achieved / peaks, 4),
                     "traffic": None if traffic is None else round(traffic, 0),
                     "alg_bytes_per_launch": alg[dom], "launch_ms": round(ms, 4),
                     "peak_source": peak_src},
        "stages_ms": {k: round(v, 4) for k, v in stages.items()} | {"sgd_epoch": round(sgd_ms, 4)},
        "step_share_ms": {k: round(v, 2) for k, v in share.items()},
        "fft_pass": {"alg_bytes": fft_pass_bytes, "ms": round(fft_pass_ms, 4),
                     "achieved_gbs": round(fft_pass_bytes / (fft_pass_ms * 1e-3) / 1e9, 1),
                     "frac": round(fft_pass_bytes / (fft_pass_ms * 1e-3) / 1e9 / peaks, 4)},
        "grid": {"n_boxes": nb_, "N": N, "M": M},
    }


def measured_traffic(stage, n):
    """DRAM bytes per launch of a stage from the committed ncu summary (profiles/dram_traffic_hybrid_1m.md),
    scaled to this run's size; None when the stage was not captured"""
    path = os.path.join(ROOT, "profiles", "dram_traffic_hybrid_1m.md")
    try:
        text = open(path).read()
    except OSError:
        return None
    block = text.split("```traffic", 1)[-1].split("```", 1)[0] if "```traffic" in text else ""
    for line in block.splitlines():
        f = line.split()
        if len(f) == 4 and f[0] == stage and f[2] == "n":
            return float(f[1]) * n / float(f[3])
    return None


def measured_peak():
    """(HBM GB/s, where it came from): the pool's measured copy bandwidth when MEASURED_PEAKS.json is present, else
    the earlier measurement of this pool's B200s (6,650 GB/s)"""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (of measured)"
    except (OSError, KeyError, ValueError):
        return 6650.0, "6650 GB/s, an earlier copy measurement on this pool (of fallback)"


# ----------------------------------------------------------------------------------------------- FFT pass alone
def fft_grid_bench(n_boxes, steps, warmup, n=300_000, seed=0):
    """The FFT pass (spread, forward rows, column convolution, inverse rows, gather + step) at a given grid: n points
    spread uniformly over a square of n_boxes boxes of width 0.7 (so the reference's grid rule picks that grid), a
    random symmetric affinity matrix of 8 entries per row; per-stage CUDA-event times of the device loop over
    `steps` iterations after `warmup`, with each stage's algorithmic bytes and achieved GB/s. The small case that
    the per-kernel ncu captures run on (about 1.3 GB on the device at 708 boxes)."""
    import torch
    import scipy.sparse as sp
    import magnet_b200 as mg
    rng = np.random.default_rng(seed)
    side = n_boxes * 0.7 - 0.01
    Y = rng.uniform(0, side, (n, 2)).astype(np.float32)
    rows = np.repeat(np.arange(n), 4)
    cols = rng.integers(0, n, rows.size)
    P = sp.csr_matrix((np.ones(rows.size, np.float32), (rows, cols)), shape=(n, n))
    P = (P + P.T).tocsr()
    P.sum_duplicates()
    P.sort_indices()
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    ip, ix, dd = t(P.indptr.astype(np.int32)), t(P.indices.astype(np.int32)), t((P.data / P.data.sum()).astype(np.float32))
    Yd = t(Y)
    if warmup:
        mg._native.optimize_tsne_profiled(ip, ix, dd, Yd.clone(), warmup, 0, 12.0, 1.0, -1.0, 3, 0.7, 1.0)
    prof = mg._native.optimize_tsne_profiled(ip, ix, dd, Yd.clone(), steps, 0, 12.0, 1.0, -1.0, 3, 0.7, 1.0)
    nb, N, M, Mh = prof["grid"]
    nnz = int(P.nnz)
    alg = {"spread": 8.0 * n + 12.0 * N * N, "row_fwd": 12.0 * N * N + 24.0 * N * Mh,
           "col_conv": 48.0 * N * Mh + 8.0 * M * Mh, "row_inv": 24.0 * N * Mh + 12.0 * N * N,
           "gather_attr_step": 12.0 * N * N + 8.0 * n + 16.0 * nnz + 68.0 * n}
    peak, src = measured_peak()
    out = {"metric": "FFT pass stages at a fixed grid", "unit": "ms", "n_points": n, "nnz": nnz, "steps": steps,
           "warmup": warmup, "grid": {"n_boxes": nb, "N": N, "M": M}, "peak_gbs": peak, "peak_source": src,
           "stages": {}}
    for k in ("bbox_grid", "twiddles", "spectra", "spread", "row_fwd", "col_conv", "row_inv", "gather_attr_step"):
        ms = prof[k] / steps
        st = {"ms": round(ms, 4)}
        if k in alg:
            st["alg_bytes"] = alg[k]
            st["gbs"] = round(alg[k] / (ms * 1e-3) / 1e9, 1)
            st["frac"] = round(alg[k] / (ms * 1e-3) / 1e9 / peak, 4)
        out["stages"][k] = st
    fp = ("spread", "row_fwd", "col_conv", "row_inv")
    fms = sum(prof[k] for k in fp) / steps
    fb = sum(alg[k] for k in fp)
    out["fft_pass"] = {"ms": round(fms, 4), "alg_bytes": fb, "gbs": round(fb / (fms * 1e-3) / 1e9, 1),
                       "frac": round(fb / (fms * 1e-3) / 1e9 / peak, 4)}
    print(json.dumps(out))


# ----------------------------------------------------------------------------------------------- fuzzy graph
def spectral_inputs(P, n_components=2, seed=0):
    """the arguments magnet/spectral.py:14-31 builds for chebyshev_eigenvectors"""
    import scipy.sparse as sp
    from scipy.sparse.csgraph import connected_components
    P = sp.csr_matrix(P, dtype=np.float32)
    deg = np.asarray(P.sum(1)).ravel().astype(np.float64)
    sd = np.where(deg > 0, 1.0 / np.sqrt(np.maximum(deg, 1e-12)), 0.0).astype(np.float32)
    _, comp = connected_components(P, directed=False)
    extra = max(2, n_components)
    X = np.random.default_rng(seed).standard_normal((P.shape[0], n_components + extra)).astype(np.float32)
    degree = 30
    max_iter = int(max(3, min(25, int(3e9 / max(1, P.nnz * (n_components + extra) * degree)))))
    return (P.indptr.astype(np.int32), P.indices.astype(np.int32), P.data.astype(np.float32), X, sd,
            comp.astype(np.int32), n_components, degree, max_iter, 0.05)


def spectral_bench(n, steps, warmup, cpu_baseline=True):
    """The spectral initialisation's solver (chebyshev_eigenvectors, src/spectral.cpp:141-241, with the arguments
    of magnet/spectral.py) on the workload's fuzzy graph: the device solver on device-resident arrays (CUDA
    events), through host arrays (end to end), and the reference's compiled solver on all host threads, with the
    largest principal-angle sine between the two results' leading vectors. One JSON line."""
    import torch
    from magnet_b200 import _native as N
    w = make_workload(n)
    a = spectral_inputs(w["P"])
    dev = torch.device("cuda", torch.cuda.current_device())
    t = lambda x: torch.from_numpy(np.ascontiguousarray(x)).to(dev)
    ad = [t(a[0]), t(a[1]), t(a[2]), None, t(a[4]), t(a[5])]
    X0 = t(a[3])
    times, e2e = [], []
    Xd = None
    for i in range(warmup + steps):
        Xd = X0.clone()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        N.chebyshev_eigenvectors(ad[0], ad[1], ad[2], Xd, ad[4], ad[5], *a[6:], -1)
        e1.record()
        torch.cuda.synchronize()
        h0 = time.perf_counter()
        N.chebyshev_eigenvectors(*a[:3], a[3].copy(), *a[4:], -1)
        h1 = time.perf_counter()
        if i >= warmup:
            times.append(e0.elapsed_time(e1) / 1000)
            e2e.append(h1 - h0)
    out = {"metric": "spectral init solver s (chebyshev_eigenvectors, %d x %d block)" % a[3].shape, "unit": "s",
           "higher_is_better": False, "steps": steps, "warmup": warmup, "dtype": "f64",
           "config": {"workload": "the fuzzy graph of the %d-point hybrid workload" % n, "nnz": int(w["P"].nnz),
                      "degree": a[7], "max_iter": a[8]},
           "value": round(statistics.median(times), 5), "e2e": {"value": round(statistics.median(e2e), 5), "unit": "s"}}
    if cpu_baseline:
        from oracle import oracle as O
        R = O.reference()
        if R is not None:
            h0 = time.perf_counter()
            Xr = np.asarray(R.chebyshev_eigenvectors(*a[:3], a[3].copy(), *a[4:], -1))
            ref_s = time.perf_counter() - h0
            qa, _ = np.linalg.qr(Xd.cpu().numpy()[:, :2].astype(np.float64))
            qb, _ = np.linalg.qr(Xr[:, :2].astype(np.float64))
            cos = np.clip(np.linalg.svd(qa.T @ qb, compute_uv=False), 0.0, 1.0)
            out["cpu_baseline"] = {"value": round(ref_s, 3), "unit": "s", "cores": os.cpu_count(), "kind": "reference",
                                   "sample": "one whole call of the reference's compiled solver on the same inputs"}
            out["subspace_sine"] = float(np.sqrt(max(0.0, 1.0 - cos.min() ** 2)))
    print(json.dumps(out))


def graph_bench(n, steps, warmup, cpu_baseline=True):
    """The fuzzy neighbour graph of the workload (smooth_knn + fuzzy union, magnet/knn.py:215-230) on the device:
    device-resident passes timed with CUDA events through the C ABI, the package's fuzzy_graph on host arrays
    (end to end), and the reference's own CPU path (its compiled smooth_knn on all host threads, then the scipy
    union of magnet/knn.py:221-230) on the same kNN. One JSON line."""
    import ctypes
    import torch
    import scipy.sparse as sp
    from magnet_b200 import graph as G
    X, _ = make_data(n, seed=2)
    ind, dist = G.exact_knn(X, 15)
    ind = np.ascontiguousarray(ind, dtype=np.int32)
    dist = np.ascontiguousarray(dist, dtype=np.float32)
    k = ind.shape[1]
    lib = ctypes.CDLL(os.path.join(ROOT, "lib-magnet_b200", "libmagnet_b200.so"))
    P_, I64 = ctypes.c_void_p, ctypes.c_int64
    lib.mg_smooth_knn.argtypes = [P_, I64, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_int, P_]
    lib.mg_fuzzy_union.argtypes = [P_, P_, I64, ctypes.c_int, I64, ctypes.c_double, P_, P_, P_, I64,
                                   ctypes.POINTER(I64)]
    lib.mg_launch_count.restype = ctypes.c_uint64
    dev = torch.device("cuda", torch.cuda.current_device())
    dd, idd = torch.from_numpy(dist).to(dev), torch.from_numpy(ind).to(dev)
    vd = torch.empty_like(dd)
    cap = 2 * n * k
    ipd = torch.empty(n + 1, dtype=torch.int32, device=dev)
    ixd = torch.empty(cap, dtype=torch.int32, device=dev)
    dtd = torch.empty(cap, dtype=torch.float32, device=dev)
    nnz = I64(0)

    def device_pass():
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        torch.cuda.synchronize()
        ev[0].record()
        if lib.mg_smooth_knn(dd.data_ptr(), n, k, 15, 1.0, 64, vd.data_ptr()) != 0:
            raise RuntimeError("mg_smooth_knn failed")
        ev[1].record()
        if lib.mg_fuzzy_union(idd.data_ptr(), vd.data_ptr(), n, k, n, 1.0, ipd.data_ptr(), ixd.data_ptr(),
                              dtd.data_ptr(), cap, ctypes.byref(nnz)) != 0:
            raise RuntimeError("mg_fuzzy_union failed")
        ev[2].record()
        torch.cuda.synchronize()
        return ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2])

    for _ in range(warmup):
        device_pass()
    l0 = lib.mg_launch_count()
    times = [device_pass() for _ in range(steps)]
    launches = int(lib.mg_launch_count() - l0) // max(steps, 1)
    smooth_ms = statistics.median(t[0] for t in times)
    union_ms = statistics.median(t[1] for t in times)
    e2e_s = float("inf")
    for _ in range(2):   # the first call also sizes the staging buffers
        t0 = time.perf_counter()
        P = G.fuzzy_graph(ind, dist, 15)
        e2e_s = min(e2e_s, time.perf_counter() - t0)
    out = {"metric": "fuzzy neighbour graph (smooth_knn + union) ms", "n": n, "k": k, "nnz": int(nnz.value),
           "value": round(smooth_ms + union_ms, 3), "unit": "ms", "smooth_knn_ms": round(smooth_ms, 3),
           "union_ms": round(union_ms, 3), "e2e": {"value": round(e2e_s * 1e3, 2), "unit": "ms"},
           "gpu_launches": launches, "steps": steps, "warmup": warmup, "higher_is_better": False,
           "data": "synthetic", "config": {"workload": "15-NN fuzzy graph of the hybrid workload's data (n=%d, d=50, "
                                                       "100 anisotropic Gaussians, seed 2), exact kNN" % n}}
    if cpu_baseline:
        from oracle import oracle as O
        R = O.reference()
        if R is not None:
            t0 = time.perf_counter()
            vals = np.asarray(R.smooth_knn(dist, 15, 1.0, 64, -1))
            t1 = time.perf_counter()
            rows = np.repeat(np.arange(n, dtype=np.int64), k)
            A = sp.csr_matrix((vals.ravel(), (rows, ind.ravel())), shape=(n, n), dtype=np.float32)
            A.eliminate_zeros()
            T = A.T.tocsr()
            prod = A.multiply(T)
            Pr = (1.0 * (A + T - prod) + 0.0 * prod).tocsr()
            Pr.eliminate_zeros()
            Pr.sort_indices()
            t2 = time.perf_counter()
            out["cpu_baseline"] = {"value": round((t2 - t0) * 1e3, 1), "unit": "ms", "cores": os.cpu_count(),
                                   "kind": "reference", "smooth_knn_ms": round((t1 - t0) * 1e3, 1),
                                   "union_ms": round((t2 - t1) * 1e3, 1),
                                   "sample": "the whole graph: the reference's compiled smooth_knn on all host "
                                             "threads, then magnet/knn.py's scipy union"}
            out["parity"] = {"pattern_equal": bool(np.array_equal(P.indptr, Pr.indptr)
                                                   and np.array_equal(P.indices, Pr.indices)),
                             "max_abs_diff": float(np.abs(P.data - Pr.data).max())}
    print(json.dumps(out), flush=True)


# ----------------------------------------------------------------------------------------------- served form
def serve_workload(n=200_000, d=64, centers=50, seed=3):
    """the served layout's data: a 50-Gaussian mixture in d = 64 (Dirichlet(1) weights, means N(0, 6^2), unit
    covariance), seed 3; returns the rows and a sampler of new rows from the same mixture"""
    rng = np.random.default_rng(seed)
    wts = rng.dirichlet(np.ones(centers))
    C = rng.normal(0, 6.0, (centers, d))

    def draw(m, r):
        return (C[r.choice(centers, m, p=wts)] + r.normal(0, 1, (m, d))).astype(np.float32)
    return draw(n, rng), draw


def serve_stream(draw, n_requests, rate, fit_sizes, seed):
    """the request stream of the served form: sizes uniform in [1, 4096], Poisson gaps at `rate`, the batches
    and the fit requests' rows (submitted right after the transform request they are keyed by)"""
    rng = np.random.default_rng(seed + 1)
    sizes = rng.integers(1, 4097, n_requests)
    gaps = rng.exponential(1.0 / rate, n_requests)
    batches = [draw(int(m), rng) for m in sizes]
    fit_at = dict(zip(sorted(rng.choice(np.arange(1, n_requests), len(fit_sizes), replace=False).tolist()),
                      [draw(f, rng) for f in fit_sizes]))
    return sizes, gaps, batches, fit_at


def transform_knn15(X_train, Y_train, X_new, Y_new, k=15, limit=3000):
    """15-NN preservation of transformed rows: each new row's k nearest training rows in the data against the k
    nearest training rows of its layout position (the first `limit` new rows), mean overlap / k"""
    from sklearn.neighbors import NearestNeighbors
    from scipy.spatial import cKDTree
    Xn, Yn = np.asarray(X_new[:limit]), np.asarray(Y_new[:limit], dtype=np.float64)
    hi = NearestNeighbors(n_neighbors=k, algorithm="brute", n_jobs=-1).fit(X_train).kneighbors(
        Xn, return_distance=False)
    lo = cKDTree(np.asarray(Y_train, dtype=np.float64)).query(Yn, k, workers=-1)[1]
    return float(np.mean([len(np.intersect1d(a, b)) / k for a, b in zip(hi, lo)]))


def reference_serve(n_requests=300, rate=200.0, fit_sizes=(5000, 20000, 50000), seed=3, n_train=200_000):
    """The served workload on the reference's CPU path (its compiled module on all host threads, driven as
    MAGNET.fit / MAGNET.transform drive it): the same fitted 200k x 64 layout, built by the reference, and the
    same request stream. The reference has no server, so requests run one at a time in arrival order: each starts
    at max(its arrival, the previous request's end), with processing times measured."""
    from oracle import oracle as O
    if O.reference() is None:
        return {"transform": {"unavailable": "the reference module (oracle/_ref) is not built"}}
    t0 = time.perf_counter()
    X, draw = serve_workload(n=n_train, seed=seed)
    a, b = O.find_ab_params(1.0, 0.1)
    Y, P = O.reference_fit(X, n_epochs=200, seed=0, a=a, b=b)
    landmarks = O.choose_landmarks(n_train, 0)
    step = O.transform_step(Y)
    setup_s = time.perf_counter() - t0
    sizes, gaps, batches, fit_at = serve_stream(draw, n_requests, rate, fit_sizes, seed)
    arrivals = np.cumsum(gaps)
    clock = 0.0
    lat_t, lat_f = [], []
    placed = []
    for i in range(n_requests):
        start = max(arrivals[i], clock)
        t = time.perf_counter()
        placed.append(O.reference_transform(X, P, Y, landmarks, step, batches[i], a=a, b=b, n_epochs=100, seed=i))
        clock = start + (time.perf_counter() - t)
        lat_t.append(clock - arrivals[i])
        if i in fit_at:
            start = max(arrivals[i], clock)
            t = time.perf_counter()
            O.reference_fit(fit_at[i], n_epochs=200, seed=0, a=a, b=b)
            clock = start + (time.perf_counter() - t)
            lat_f.append(clock - arrivals[i])
    span = clock - arrivals[0]

    def summary(lat, pts):
        lat = np.asarray(lat) * 1e3
        return {"requests": len(lat), "p50_ms": round(float(np.percentile(lat, 50)), 2),
                "p99_ms": round(float(np.percentile(lat, 99)), 2), "mean_ms": round(float(lat.mean()), 2),
                "points_per_s": round(pts / max(span, 1e-9), 2)}
    knn15 = transform_knn15(X, Y, np.concatenate(batches), np.concatenate(placed))
    return {"transform": summary(lat_t, int(sizes.sum())) | {"slots": 1, "knn15": round(knn15, 4)},
            "fit_requests": summary(lat_f, int(sum(len(v) for v in fit_at.values()))),
            "serve_config": {"layout": "200,000 x 64, 50-Gaussian mixture, seed 3, k=15 (built by the reference)",
                             "requests": n_requests, "rate_per_s": rate, "batch": "uniform integer [1, 4096]",
                             "transform_epochs": 100, "fits": list(fit_sizes), "cores": os.cpu_count(),
                             "server": "one request at a time in arrival order", "setup_s": round(setup_s, 1)}}


def serve_bench(n_requests=300, rate=200.0, slots=4, fit_sizes=(5000, 20000, 50000), seed=3, dist=None):
    """The served form: a fitted 200k x 64 layout resident on the device; transform() requests of 1-4096 new rows
    from the same mixture with Poisson arrivals at `rate` per second (100 SGD epochs each, the training rows
    fixed), interleaved with fit requests of 5k-50k rows. Run once on one slot (the plain form: one request at a
    time) and once on `slots` slots (continuous batching); latency is submit to result. With several ranks every
    rank keeps its own resident copy of the layout, the requests are placed on the ranks by free device memory
    (magnet_b200.replicas.place, the same placement on every rank) and each rank serves its share; the latencies
    and placed rows are gathered, and the summary covers the whole stream."""
    from magnet_b200 import serve as S
    from magnet_b200 import replicas as Rp
    import magnet_b200 as mg
    t0 = time.perf_counter()
    X, draw = serve_workload(seed=seed)
    Y, P = S.fit_layout(X, n_epochs=200, seed=0, return_graph=True)
    a, b = mg.find_ab_params(1.0, 0.1)
    layout = S.FittedLayout(X, Y, a=a, b=b, transform_epochs=100, graph=P)
    setup_s = time.perf_counter() - t0
    sizes, gaps, batches, fit_at = serve_stream(draw, n_requests, rate, fit_sizes, seed)
    big = batches[int(np.argmax(sizes))]
    # the stream in submission order: (arrival index, kind, rows) and each request's device bytes
    stream = []
    for i in range(n_requests):
        stream.append((i, "transform", batches[i]))
        if i in fit_at:
            stream.append((i, "fit", fit_at[i]))
    nbytes = [layout.request_bytes(len(r)) if k == "transform" else S.fit_bytes(len(r), X.shape[1])
              for _, k, r in stream]
    rank = 0 if dist is None else dist.get_rank()
    owner = Rp.place(nbytes, Rp.free_bytes(dist, budget_fraction=0.5))

    def run(k):
        srv = S.device_server(layout, slots=k)
        warm = [srv.submit("transform", (big, 0), layout.request_bytes(len(big)), len(big)) for _ in range(k)]
        warm.append(srv.submit("fit", fit_at[min(fit_at)], S.fit_bytes(len(fit_at[min(fit_at)]), X.shape[1]), 0))
        for f in warm:
            f.result()
        srv.done.clear()
        if dist is not None:
            dist.barrier()
        futs = []
        t_next = time.perf_counter()
        last = -1
        for j, (i, kind, rows) in enumerate(stream):
            if i != last:   # the arrival of request i (a fit arrives with the transform it is keyed by)
                t_next += gaps[i]
                last = i
            if owner[j] != rank:
                continue
            dt = t_next - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
            payload = (rows, i) if kind == "transform" else rows
            futs.append((j, kind, srv.submit(kind, payload, nbytes[j], len(rows))))
        res = [(j, kind, f.result()) for j, kind, f in futs]
        srv.close()
        recs = [(r.kind, r.t_submit, r.t_done, r.points) for r in srv.done]
        placed = [(j, y) for j, kind, y in res if kind == "transform"]
        if dist is not None:
            allrecs = [None] * dist.get_world_size()
            dist.all_gather_object(allrecs, recs)
            recs = [r for part in allrecs for r in part]
        placed = Rp.gather_results(placed, dist)
        tr, fi = summarise(recs, "transform"), summarise(recs, "fit")
        order = [j for j, (_, kind, _) in enumerate(stream) if kind == "transform"]
        X_new = np.concatenate([stream[j][2] for j in order])
        tr["knn15"] = transform_knn15(X, Y, X_new, np.concatenate(placed))
        return {k2: round(v, 4 if k2 == "knn15" else 2) for k2, v in tr.items()}, \
            {k2: round(v, 1) for k2, v in fi.items()}

    plain, plain_fit = run(1)
    mixed, mixed_fit = run(slots)
    world = 1 if dist is None else dist.get_world_size()
    return {"transform": mixed | {"slots": slots}, "transform_plain": plain | {"slots": 1},
            "fit_requests": {"mixed": mixed_fit, "plain": plain_fit},
            "serve_config": {"layout": "200,000 x 64, 50-Gaussian mixture, seed 3, k=15, resident%s" %
                                       (" on each of %d GPUs" % world if world > 1 else ""),
                             "requests": n_requests, "rate_per_s": rate, "batch": "uniform integer [1, 4096]",
                             "transform_epochs": 100, "fits": list(fit_sizes), "mode": "owner",
                             "query_knn": "beam search over the training graph (device)",
                             "placement": "by free HBM over %d rank(s)" % world, "setup_s": round(setup_s, 1)}}


def summarise(recs, kind):
    """p50 / p99 / mean latency (ms) and points/s of the (kind, t_submit, t_done, points) records of one kind"""
    rs = [r for r in recs if r[0] == kind]
    if not rs:
        return {}
    lat = np.array([(r[2] - r[1]) * 1e3 for r in rs])
    span = max(r[2] for r in rs) - min(r[1] for r in rs)
    return {"requests": len(rs), "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "points_per_s": float(sum(r[3] for r in rs) / max(span, 1e-9))}


# ----------------------------------------------------------------------------------------------- ranks
def max_over_ranks(x, dist=None, device="cpu"):
    """the largest of x over the ranks (the job's time is its slowest rank's); every rank takes the same
    collective step, NCCL on the GPU path, gloo in the host tests"""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def seconds_per_layout(ms_max, n_ranks):
    """the whole job's seconds per layout: each rank lays out one replica per step, so the job finishes
    n_ranks layouts in the slowest rank's step time"""
    return ms_max / 1000.0 / n_ranks


# ----------------------------------------------------------------------------------------------- main
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="magnet_b200", choices=["magnet_b200", "reference"])
    ap.add_argument("--n", type=int, default=1_000_000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--graph", action="store_true", help="time the fuzzy neighbour graph instead of the layout")
    ap.add_argument("--no-serve", action="store_true", help="skip the served-form measurement")
    ap.add_argument("--spectral", action="store_true", help="time the spectral initialisation's solver")
    ap.add_argument("--serve-requests", type=int, default=300)
    ap.add_argument("--fft-grid", type=int, default=0, help="time the FFT pass alone at this many boxes per side")
    ap.add_argument("--config", type=int, default=3, choices=[1, 2, 3, 4],
                    help="1: the 10k umap layout, 2: the 70k tsne layout, 3 (default): the 1M hybrid layout, "
                         "4: 256 batched t-SNE layouts")
    args = ap.parse_args()
    if args.fft_grid:
        import torch
        torch.cuda.set_device(0)
        fft_grid_bench(args.fft_grid, args.steps, args.warmup)
        return
    if args.config in (1, 2, 4):
        if args.impl != "reference":
            import torch
            torch.cuda.set_device(0)
        if args.config == 4:
            config4_leg(args.impl, args.steps, args.warmup)
        else:
            config_leg(args.config, args.impl, args.steps, args.warmup)
        return
    if args.graph:
        import torch
        torch.cuda.set_device(0)
        graph_bench(args.n, args.steps, args.warmup, not args.no_cpu_baseline)
        return
    if args.spectral:
        import torch
        torch.cuda.set_device(0)
        spectral_bench(args.n, args.steps, args.warmup, not args.no_cpu_baseline)
        return

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    # the same config in both arms (the graph each arm builds is named in "inputs")
    config = {"workload": "hybrid layout, n=%d, d=50, 100 anisotropic Gaussians, seed 2, k=15, %d SGD epochs + %d "
                          "FFT iterations" % (args.n, N_EPOCHS, HYBRID_ITER),
              "n_points": args.n, "l2": "inputs larger than L2 (126 MB): about 24 edges per point, 20 B each",
              "init": "PCA (spectral stand-in)", "parallelism": "replicas %d" % world}

    if args.impl == "reference":
        # the reference's CPU path needs no GPU and no process group: rank 0 alone runs it, the others exit
        if rank != 0:
            return
        nt = os.cpu_count() or 1
        w = make_workload_reference(args.n, n_threads=-1)
        rp = ReferencePass(w, args.steps, -1)
        for _ in range(args.warmup):
            rp.warmup()
        times = []
        Y_ref = None
        for j in range(args.steps):
            t0 = time.perf_counter()
            Y_ref = rp.piece(j)
            times.append(time.perf_counter() - t0)
        value = sum(times)
        knn15 = knn_preservation(w["X"], Y_ref)
        sample = ("the whole pass, timed in %d consecutive pieces: piece 1 the 200-epoch SGD call and the rescale "
                  "(%.2f s), pieces 2-%d the 300 full-batch iterations (%.2f s); the reference's compiled module on "
                  "all %d host threads" % (args.steps, times[0], args.steps, sum(times[1:]), nt)) \
            if args.steps > 1 else "the whole pass in one step on all %d host threads" % nt
        line = {"impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(value * 1000 / args.steps, 1),
                "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic", "config": config,
                "inputs": {"graph": w["graph"], "edges": int(w["head"].size), "setup_s": round(w["setup_s"], 1)},
                "knn15": round(knn15, 4),
                "pass_s": {"sgd_and_rescale": round(times[0], 3), "tsne": round(sum(times[1:]), 3)},
                "cpu_baseline": {"value": round(value, 3), "unit": "s", "cores": nt, "kind": "reference",
                                 "sample": sample},
                "e2e": {"value": round(value, 3), "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        if not args.no_serve:
            try:
                line.update(reference_serve(n_requests=args.serve_requests))
            except Exception as e:  # noqa: BLE001  (the layout's line is reported either way)
                line["transform"] = {"error": "%s: %s" % (type(e).__name__, e)}
        print(json.dumps(line))
        return

    import torch
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    else:
        torch.cuda.set_device(0)

    import magnet_b200 as mg
    w = make_workload(args.n)
    gp = GpuPass(w)
    for _ in range(args.warmup):
        gp.step_device()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    st = torch.cuda.current_stream()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = mg.launch_count()
    with Clocks(local) as clk:
        ev0.record(st)
        for _ in range(args.steps):
            gp.step_device()
        ev1.record(st)
        torch.cuda.synchronize()
    launches = mg.launch_count() - launches0
    ms = max_over_ranks(ev0.elapsed_time(ev1) / args.steps, dist, "cuda")
    Y_final = gp.result()

    # end-to-end through the reference-shaped API with pinned host arrays
    gp.step_e2e()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(max(1, min(args.steps, 3))):
        h2d, d2h = gp.step_e2e()
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1000 / max(1, min(args.steps, 3)), dist, "cuda")

    rf = roofline(w, gp, measured_peak())
    knn15 = knn_preservation(w["X"], Y_final)
    precision = precision_study(Y_final)
    n_gpus = world
    line = {"metric": METRIC, "value": round(seconds_per_layout(ms, n_gpus), 4), "unit": "s", "n_gpus": n_gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 2), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config,
            "inputs": {"graph": w["graph"], "edges": int(w["head"].size), "setup_s": round(w["setup_s"], 1)},
            "knn15": round(knn15, 4), "grid": rf["grid"], "precision": precision,
            "e2e": {"value": round(seconds_per_layout(e2e_ms, n_gpus), 4), "unit": "s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": int(launches), "clocks": clk.summary(), "roofline": rf["roofline"],
            "fft_pass": rf["fft_pass"], "stages_ms": rf["stages_ms"], "step_share_ms": rf["step_share_ms"]}
    if rank == 0 and n_gpus == 1 and not args.no_cpu_baseline:
        try:
            v, nt, sample = reference_sample(w, Y_tsne=Y_final, sgd_epochs=4, tsne_iters=4)
            line["cpu_baseline"] = {"value": round(v, 2), "unit": "s", "cores": nt, "kind": "reference",
                                    "sample": sample}
        except Exception as e:  # noqa: BLE001
            line["cpu_baseline"] = {"value": None, "unit": "s", "cores": os.cpu_count(), "kind": "reference",
                                    "sample": "unavailable: %s" % e}
    if not args.no_serve:
        try:
            line.update(serve_bench(n_requests=args.serve_requests, dist=dist))
        except Exception as e:  # noqa: BLE001  (the layout's line is reported either way)
            line["transform"] = {"error": "%s: %s" % (type(e).__name__, e)}
    if dist is not None:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


if __name__ == "__main__":
    main()
