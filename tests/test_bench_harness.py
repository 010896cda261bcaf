"""The benchmark's host-side harness (no GPU): the t-SNE input affinities that the harness builds for the perplexity
configurations (the reference has no perplexity calibration), pinned against scikit-learn's published binary search
of the same conditional Gaussians; the synthetic data of the benchmark configurations; the whole-pass cut of the
reference arm."""
import numpy as np
import pytest
import scipy.sparse as sp

import bench


def test_perplexity_affinities_match_sklearn():
    from sklearn.manifold import _utils
    rng = np.random.default_rng(0)
    X = np.vstack([rng.normal(c, 1.0, (700, 20)) for c in (0, 4, 9)]).astype(np.float32)
    ind, d2 = bench.exact_knn_cpu(X, 90)
    P = bench.perplexity_affinities(ind, d2, 30.0)
    n = X.shape[0]
    Pc = _utils._binary_search_perplexity(d2.astype(np.float32), 30.0, 0)
    C = sp.csr_matrix((Pc.ravel(), (np.repeat(np.arange(n), 90), ind.ravel())), shape=(n, n))
    Ps = ((C + C.T) / (2.0 * n)).tocsr()
    assert abs(P.sum() - 1.0) < 1e-5
    assert abs(P - P.T).max() < 1e-9
    assert abs(P - Ps).max() <= 1e-5 * Ps.max()
    # each row's conditional distribution has the target perplexity
    Cm = C.toarray()
    H = -(Cm * np.log(np.where(Cm > 0, Cm, 1.0))).sum(1)
    assert np.allclose(np.exp(H), 30.0, rtol=1e-3)


def test_config_data_shapes_and_seeds():
    X1, y1 = bench.config1_data()
    assert X1.shape == (10_000, 50) and X1.dtype == np.float32 and set(np.unique(y1)) == set(range(10))
    assert np.array_equal(X1, bench.config1_data()[0])
    X2, _ = bench.config2_data(n=2000)
    assert X2.shape == (2000, 784) and X2.min() >= 0.0 and X2.max() <= 1.0
    img = X2.reshape(-1, 28, 28).mean(0)
    outside = np.delete(img.ravel(), [r * 28 + c for r in range(4, 24) for c in range(4, 24)])
    assert img[4:24, 4:24].mean() > 5 * outside.mean()
    sizes = [len(X) for X in bench.config4_instances(256)]
    assert min(sizes) >= 500 and max(sizes) <= 20000 and len(set(sizes)) > 200


@pytest.mark.parametrize("pieces", [1, 2, 5, 19, 300])
def test_reference_pass_pieces_cover_the_pass(pieces):
    """the reference arm's timed pieces after the SGD piece run the 300 iterations exactly once"""
    its = bench.split_iterations(bench.HYBRID_ITER, pieces)
    assert len(its) == pieces and sum(its) == bench.HYBRID_ITER and min(its) >= 1
    assert max(its) - min(its) <= 1
    assert bench.split_iterations(bench.HYBRID_ITER, 0) == []
