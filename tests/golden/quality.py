"""Layout-quality measures shared by the fixture scripts and the tests.

* ``knn_preservation``: benchmarks/metrics.py:52-62 of the reference, the k-NN preservation of a seeded query
  subsample (exact k-NN in the data, self excluded, against the layout's k-NN), mean overlap / k;
* ``kl_divergence``: KL(P || Q) of a layout, P the affinities normalised to sum 1 and Q the Student-t similarities
  (1 + |y_i - y_j|^2 / dof)^-dof normalised over all pairs i != j, in FP64 with the normaliser summed in blocks.
  The reference computes no KL (its t-SNE loop never forms it); both sides of a comparison use this one.
"""
import numpy as np
import scipy.sparse as sp


def query_rows(n, n_query=5000, seed=0):
    """the fixed query subsample of benchmarks/metrics.py:15-16"""
    return np.sort(np.random.default_rng(seed).choice(n, size=min(n_query, n), replace=False))


def high_dim_neighbors(X, k=15, n_query=5000, seed=0):
    from sklearn.neighbors import NearestNeighbors
    q = query_rows(X.shape[0], n_query, seed)
    ind = NearestNeighbors(n_neighbors=k + 1, algorithm="brute", n_jobs=-1).fit(X).kneighbors(
        X[q], return_distance=False)
    return np.array([row[row != i][:k] for i, row in zip(q, ind)])


def knn_preservation(X, Y, k=15, n_query=5000, seed=0, hnn=None):
    """hnn: the data's neighbours of the query rows when already computed (high_dim_neighbors)"""
    from scipy.spatial import cKDTree
    Y = np.asarray(Y, dtype=np.float64)
    q = query_rows(Y.shape[0], n_query, seed)
    if hnn is None:
        hnn = high_dim_neighbors(X, k, n_query, seed)
    lnn = cKDTree(Y).query(Y[q], k + 1)[1]
    lnn = np.array([row[row != i][:k] for i, row in zip(q, lnn)])
    return float(np.mean([len(np.intersect1d(a, b)) for a, b in zip(hnn, lnn)]) / k)


def kl_divergence(P, Y, dof=1.0, block=2048):
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
    keep = C.data > 0          # zero entries contribute nothing (0 log 0 = 0)
    d2 = ((Y[C.row[keep]] - Y[C.col[keep]]) ** 2).sum(-1)
    q = (1.0 + d2 / dof) ** (-dof) / Z
    p = C.data[keep]
    return float((p * np.log(p / q)).sum())
