"""The fuzzy neighbour graph on the device (smooth_knn, then the fuzzy union A + A^T - A o A^T) against the
reference's own outputs (graph_small.npz: its compiled smooth_knn and magnet/knn.py fuzzy_graph) and the oracle.
The union is bit-exact given the same memberships. The memberships come from exp in FP64 rounded to float, against
the reference's glibc expf: the two differ on about 1e-4 of float inputs by one ulp, so memberships match to 1e-5
(in (0, 1]) with the same zeros."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

MEMBERSHIP_TOL = 1e-5


def native():
    from magnet_b200 import _native
    return _native


@pytest.mark.parametrize("suffix", ["", "_e"])
def test_smooth_knn_against_reference(mg, golden, suffix):
    g = golden("graph_small.npz")
    out = native().smooth_knn(g["dist" + suffix], 15)
    ref = g["vals" + suffix]
    assert out.dtype == np.float32 and out.shape == ref.shape
    assert np.abs(out - ref).max() <= MEMBERSHIP_TOL, np.abs(out - ref).max()
    assert (out == ref).mean() > 0.99
    assert np.array_equal(out == 0, ref == 0)


@pytest.mark.parametrize("suffix,mix", [("", 1.0), ("_mix", 0.5), ("_e", 1.0)])
def test_fuzzy_union_bit_exact_given_memberships(mg, golden, suffix, mix):
    g = golden("graph_small.npz")
    ind = g["ind_e"] if suffix == "_e" else g["ind"]
    vals = g["vals_e"] if suffix == "_e" else g["vals"]
    indptr, indices, data = native().fuzzy_union(ind, vals, -1, mix)
    assert np.array_equal(indptr, g["indptr" + suffix])
    assert np.array_equal(indices, g["indices" + suffix])
    assert np.array_equal(data, g["data" + suffix])


@pytest.mark.parametrize("suffix,kw", [("", {}), ("_mix", dict(set_op_mix_ratio=0.5)),
                                       ("_rank", dict(rank_exponent=0.25)), ("_e", {})])
def test_fuzzy_graph_against_reference(mg, golden, suffix, kw):
    from magnet_b200 import graph as G
    g = golden("graph_small.npz")
    ind = g["ind_e"] if suffix == "_e" else g["ind"]
    dist = g["dist_e"] if suffix == "_e" else g["dist"]
    P = G.fuzzy_graph(ind, dist, 15, **kw)
    assert np.array_equal(P.indptr, g["indptr" + suffix]) and np.array_equal(P.indices, g["indices" + suffix])
    assert np.abs(P.data - g["data" + suffix]).max() <= 2 * MEMBERSHIP_TOL


def test_fuzzy_graph_20k_against_oracle(mg):
    """20,000 blob points, exact 15-NN: memberships against the oracle's to 1e-5; the union of the device's own
    memberships bit-exact against the oracle's union of the same, also over an n x n graph with n past the kNN
    rows and at set_op_mix_ratio 0.3"""
    from sklearn.neighbors import NearestNeighbors
    rng = np.random.default_rng(21)
    C = rng.normal(0, 4, (12, 10))
    X = (C[rng.integers(0, 12, 20000)] + rng.normal(0, 1, (20000, 10))).astype(np.float32)
    d, i = NearestNeighbors(n_neighbors=15).fit(X).kneighbors(X)
    ind = np.ascontiguousarray(i[:, 1:], dtype=np.int32)
    dist = np.ascontiguousarray(d[:, 1:], dtype=np.float32)
    vals = native().smooth_knn(dist, 15)
    vals_o = O.smooth_knn(dist, 15)
    assert np.abs(vals - vals_o).max() <= MEMBERSHIP_TOL and (vals == vals_o).mean() > 0.99
    for n, mix in ((None, 1.0), (20500, 1.0), (None, 0.3)):
        dev = native().fuzzy_union(ind, vals, -1 if n is None else n, mix)
        ora = O.fuzzy_union(ind, vals, n, mix)
        for a, b in zip(dev, ora):
            assert np.array_equal(a, b)
        assert dev[0].shape[0] == (20000 if n is None else n) + 1


def test_graph_argument_errors(mg, golden):
    g = golden("graph_small.npz")
    ind = g["ind"].copy()
    ind[7, 3] = 600
    with pytest.raises(RuntimeError, match="neighbour index out of range"):
        native().fuzzy_union(ind, g["vals"], -1, 1.0)
    with pytest.raises(RuntimeError, match="n_rows <= n"):
        native().fuzzy_union(g["ind"], g["vals"], 100, 1.0)
    with pytest.raises(RuntimeError, match="dist must be"):
        native().smooth_knn(g["dist"][0], 15)
