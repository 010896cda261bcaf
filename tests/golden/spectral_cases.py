"""Spectral-init test cases shared by the device tests and the oracle's pin: the arguments magnet/spectral.py builds
for chebyshev_eigenvectors, a graph of three connected components plus isolated nodes, and the subspace and Ritz
measures the tests compare with."""
import numpy as np
import scipy.sparse as sp
from scipy.sparse.csgraph import connected_components


def subspace_sine(A, B):
    qa, _ = np.linalg.qr(np.asarray(A, np.float64))
    qb, _ = np.linalg.qr(np.asarray(B, np.float64))
    cos = np.clip(np.linalg.svd(qa.T @ qb, compute_uv=False), 0.0, 1.0)
    return float(np.sqrt(max(0.0, 1.0 - cos.min() ** 2)))


def ritz_values(P, sd, X):
    """the Rayleigh quotients of the columns of X under M = (I + D^-1/2 P D^-1/2) / 2"""
    D = sp.diags(sd.astype(np.float64))
    M = 0.5 * (sp.identity(P.shape[0]) + D @ P.astype(np.float64) @ D)
    X = np.asarray(X, np.float64)
    return np.einsum("ij,ij->j", X, M @ X) / np.einsum("ij,ij->j", X, X)


def inputs(P, n_components, seed=0):
    """the arguments spectral_init builds (magnet/spectral.py:14-31)"""
    P = sp.csr_matrix(P, dtype=np.float32)
    n = P.shape[0]
    deg = np.asarray(P.sum(1)).ravel().astype(np.float64)
    sd = np.where(deg > 0, 1.0 / np.sqrt(np.maximum(deg, 1e-12)), 0.0).astype(np.float32)
    _, comp = connected_components(P, directed=False)
    extra = max(2, n_components)
    X = np.random.default_rng(seed).standard_normal((n, n_components + extra)).astype(np.float32)
    degree = 30
    max_iter = int(max(3, min(25, int(3e9 / max(1, P.nnz * (n_components + extra) * degree)))))
    return (P.indptr.astype(np.int32), P.indices.astype(np.int32), P.data.astype(np.float32), X, sd,
            comp.astype(np.int32), n_components, degree, max_iter, 0.05)


def three_components(seed=4):
    rng = np.random.default_rng(seed)
    blocks = []
    for size in (700, 400, 250):
        A = sp.random(size, size, density=12.0 / size, random_state=rng, dtype=np.float32)
        A = A + A.T + sp.diags(np.ones(size - 1, np.float32), 1) + sp.diags(np.ones(size - 1, np.float32), -1)
        blocks.append(A)
    blocks.append(sp.csr_matrix((5, 5), dtype=np.float32))   # five isolated nodes
    P = sp.block_diag(blocks, format="csr").astype(np.float32)
    P.data = np.abs(P.data) + 0.05
    return P
