"""Host-side inputs of the layout pass: the fuzzy neighbour graph, mid-near partners and the initial layout.

These steps are upstream of the layout pass. The fuzzy graph and the mid-near partners run on the device; the
others are restated here on the host, from the reference's behaviour, so that workloads can be built where the
reference is not installed:

* ``smooth_knn``: UMAP's per-row bandwidth search (src/graph.cpp:29-78), on the device;
* ``fuzzy_graph``: the fuzzy union A + A^T - A o A^T (magnet/knn.py:215-230), on the device;
* ``exact_knn``: exact k nearest neighbours (self excluded, sorted) by blocked matmul on a CUDA device when
  torch sees one, else numpy; it stands in for NN-descent (src/nndescent.cpp), whose output it bounds;
* ``mid_near_pairs``: PaCMAP-style partners, the second closest of n_cand random rows (src/nndescent.cpp:731-759),
  on the device with the reference's streams and distance arithmetic;
* ``initial_layout``: the reference's rescale of an initial embedding (magnet/__init__.py:444-448).
"""
import numpy as np
import scipy.sparse as sp


def smooth_knn(dist, n_neighbors, bandwidth=1.0, n_iter=64):
    """dist (n, k) sorted neighbour distances (self excluded) -> memberships (n, k) in (0, 1], on the device
    (src/graph.cpp:29-78)"""
    from . import _native
    return _native.smooth_knn(np.ascontiguousarray(dist, dtype=np.float32), int(n_neighbors), float(bandwidth),
                              int(n_iter))


def rescale_neighbor_distances(dist, power=1.0, rank_exponent=0.0):
    """the distance-profile reshaping of magnet/knn.py:201-213: d_k <- d_1 (d_k / d_1)^power, then
    d_k <- d_k k^rank_exponent"""
    dist = np.asarray(dist, dtype=np.float32)
    if power != 1.0:
        d1 = np.maximum(dist[:, :1], 1e-12)
        dist = d1 * (np.maximum(dist, 0.0) / d1) ** power
    if rank_exponent != 0.0:
        dist = dist * (np.arange(1, dist.shape[1] + 1, dtype=np.float32) ** rank_exponent)[None, :]
    return dist.astype(np.float32)


def fuzzy_graph(ind, dist, n_neighbors, n=None, set_op_mix_ratio=1.0, power=1.0, rank_exponent=0.0):
    """symmetric fuzzy neighbourhood graph (CSR float32, sorted indices) from kNN indices and distances
    (magnet/knn.py:215-230): smooth_knn memberships and the union A + A^T - A o A^T, both on the device"""
    from . import _native
    n = ind.shape[0] if n is None else int(n)
    if power != 1.0 or rank_exponent != 0.0:
        dist = rescale_neighbor_distances(dist, power, rank_exponent)
    vals = smooth_knn(dist, n_neighbors)
    indptr, indices, data = _native.fuzzy_union(np.ascontiguousarray(ind, dtype=np.int32), vals, n,
                                                float(set_op_mix_ratio))
    P = sp.csr_matrix((data, indices, indptr), shape=(n, n))
    P.has_sorted_indices = True
    return P


def exact_knn(X, k, block=2048):
    """(indices (n, k-1) int64, distances (n, k-1) float32) of the k-1 nearest other rows, sorted"""
    X = np.ascontiguousarray(X, dtype=np.float32)
    n = X.shape[0]
    kk = min(k, n)
    try:
        import torch
        cuda = torch.cuda.is_available()
    except ImportError:
        cuda = False
    if cuda:
        import torch
        prev = torch.backends.cuda.matmul.allow_tf32
        torch.backends.cuda.matmul.allow_tf32 = False
        Xd = torch.from_numpy(X).cuda()
        sq = (Xd * Xd).sum(1)
        I = np.empty((n, kk), np.int64)
        D = np.empty((n, kk), np.float32)
        for s in range(0, n, block):
            q = Xd[s:s + block]
            d2 = sq[s:s + block, None] - 2.0 * (q @ Xd.T) + sq[None, :]
            d2[torch.arange(q.shape[0], device=q.device), torch.arange(s, s + q.shape[0], device=q.device)] = float("inf")
            v, i = torch.topk(d2, kk - 1, dim=1, largest=False, sorted=True)
            I[s:s + block, :kk - 1] = i.cpu().numpy()
            D[s:s + block, :kk - 1] = torch.sqrt(torch.clamp(v, min=0.0)).cpu().numpy()
        torch.backends.cuda.matmul.allow_tf32 = prev
        return I[:, :kk - 1], D[:, :kk - 1]
    sq = (X.astype(np.float64) ** 2).sum(1)
    I = np.empty((n, kk - 1), np.int64)
    D = np.empty((n, kk - 1), np.float32)
    for s in range(0, n, block):
        d2 = sq[s:s + block, None] - 2.0 * (X[s:s + block].astype(np.float64) @ X.T.astype(np.float64)) + sq[None, :]
        d2[np.arange(d2.shape[0]), np.arange(s, s + d2.shape[0])] = np.inf
        part = np.argpartition(d2, kk - 1, axis=1)[:, :kk - 1]
        pd = np.take_along_axis(d2, part, 1)
        o = np.argsort(pd, 1)
        I[s:s + block] = np.take_along_axis(part, o, 1)
        D[s:s + block] = np.sqrt(np.maximum(np.take_along_axis(pd, o, 1), 0)).astype(np.float32)
    return I, D


def mid_near_pairs(X, n_pairs=5, n_cand=6, seed=0, n_threads=-1):
    """(n, n_pairs) int32 PaCMAP-style partners on the device (magnet/roles.py:36-51 over src/nndescent.cpp:731-768):
    for every row and pair, the second closest of n_cand rows drawn with the reference's streams for n_threads
    threads (-1: the host's hardware threads, as the reference resolves it), so the partners are the reference's
    own for the same thread count"""
    from . import _native
    return _native.mid_near_pairs_dense(np.ascontiguousarray(X, dtype=np.float32), int(n_pairs), int(n_cand),
                                        int(seed), int(n_threads))


def pca2(X, seed=0):
    """2-D PCA projection (randomised range finder; the t-SNE mode's init)"""
    X = np.asarray(X, dtype=np.float32)
    Xc = X - X.mean(0)
    rng = np.random.default_rng(seed)
    G = rng.normal(size=(X.shape[1], 8)).astype(np.float32)
    Q, _ = np.linalg.qr(Xc @ G)
    for _ in range(2):
        Q, _ = np.linalg.qr(Xc @ (Xc.T @ Q))
    B = Q.T @ Xc
    _, _, Vt = np.linalg.svd(B, full_matrices=False)
    return (Xc @ Vt[:2].T).astype(np.float32)


def initial_layout(Y, seed=0):
    """centred, scaled to max-abs 10, plus N(0, 1e-4) jitter (magnet/__init__.py:444-448)"""
    Y = np.array(Y, dtype=np.float32)
    Y -= Y.mean(0)
    scale = np.abs(Y).max()
    if scale > 0:
        Y *= 10.0 / scale
    Y += np.random.default_rng(seed).normal(0, 1e-4, Y.shape).astype(np.float32)
    return np.ascontiguousarray(Y, dtype=np.float32)
