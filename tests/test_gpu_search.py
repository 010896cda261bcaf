"""Query kNN on the device (knn_search, src/nndescent.cpp:585-690, the beam search of MAGNET.transform) against the
reference's own compiled knn_search on the same training rows, neighbour graph, landmarks and queries: the same
neighbours and the same squared distances, bit for bit, wherever no two distances tie."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def served(ref):
    if ref is None:
        pytest.skip("reference module not built")
    rng = np.random.default_rng(3)
    C = rng.normal(0, 6, (30, 64))
    w = rng.dirichlet(np.ones(30))
    draw = lambda m: (C[rng.choice(30, m, p=w)] + rng.normal(0, 1, (m, 64))).astype(np.float32)
    X = draw(20000)
    ind, d2 = ref.nn_descent(X, 20, 50, 10, 0.001, 4, 30, 0, -1, False)
    ind = np.asarray(ind)[:, :14].astype(np.int64)
    dist = np.sqrt(np.maximum(np.asarray(d2)[:, :14], 0.0)).astype(np.float32)
    P = O.reference_fuzzy_graph(ind, dist, 15)
    return X, P, O.choose_landmarks(20000, 0), draw(700)


def compare(got, want):
    gi, gd = got
    wi, wd = np.asarray(want[0]), np.asarray(want[1])
    same_rows = np.mean([np.array_equal(a, b) for a, b in zip(gi, wi)])
    assert same_rows >= 0.998, same_rows
    eq = gi == wi
    assert np.array_equal(gd[eq], wd[eq])
    return same_rows


def test_search_matches_reference_with_landmarks(mg, ref, served):
    X, P, land, Q = served
    gptr, gidx = P.indptr.astype(np.int32), P.indices.astype(np.int32)
    got = mg._native.knn_search(X, gptr, gidx, land, Q, 14, 64, 5, 0, -1)
    want = ref.knn_search(X, gptr, gidx, land, Q, 14, 64, 5, 0, -1)
    print("identical rows: %.4f" % compare(got, want))


def test_search_matches_reference_random_entries(mg, ref, served):
    X, P, _, Q = served
    gptr, gidx = P.indptr.astype(np.int32), P.indices.astype(np.int32)
    none = np.zeros(0, np.int32)
    got = mg._native.knn_search(X, gptr, gidx, none, Q, 10, 40, 8, 11, 3)
    want = ref.knn_search(X, gptr, gidx, none, Q, 10, 40, 8, 11, 3)
    print("identical rows: %.4f" % compare(got, want))


def test_search_device_arrays_and_rules(mg, ref, served):
    import torch
    X, P, land, Q = served
    gptr, gidx = P.indptr.astype(np.int32), P.indices.astype(np.int32)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    got = mg._native.knn_search(t(X), t(gptr), t(gidx), t(land), t(Q[:100]), 14, 64, 5, 0, -1)
    want = ref.knn_search(X, gptr, gidx, land, Q[:100], 14, 64, 5, 0, -1)
    compare(got, want)
    with pytest.raises(RuntimeError, match="need 1 <= k <= n and ef >= k"):
        mg._native.knn_search(X, gptr, gidx, land, Q, 14, 10, 5, 0, -1)
    with pytest.raises(RuntimeError, match="landmark out of range"):
        mg._native.knn_search(X, gptr, gidx, np.array([0, 20000], np.int32), Q, 14, 64, 5, 0, -1)
    with pytest.raises(RuntimeError, match="same width"):
        mg._native.knn_search(X, gptr, gidx, land, Q[:, :10], 14, 64, 5, 0, -1)
