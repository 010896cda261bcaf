"""Owner mode (optimize_layout parallel=1) on the device against the reference's own runs (sgd_owner.npz) and the
oracle. Cases with the power kernel at b = rep_b = 1 and the sgd optimizer (only +, *, / and sqrt) equal the
reference bit for bit: the layout, eons and eonns, over 2 and 23 chunks, with reverse mid pairs, walks, jumps,
fixed nodes, norm clipping, dims 2, 3 and 8, and distance-0 jitter draws (the serial fallback). Cases through
powf / expf / tanhf match the oracle to FP32 rounding after one epoch and the reference's layout quality after 40."""
import numpy as np
import pytest

import sgd_cases as C
from oracle import oracle as O

pytestmark = pytest.mark.gpu

EXACT = [c for c in C.OWNER_CASES if c.startswith("b1")]
CLOSE = [c for c in C.OWNER_CASES if not c.startswith("b1")]


@pytest.fixture(scope="module")
def big_graph():
    return C.synthetic_graph()


def run_owner(mg, g, case, big, seed=12345, stream_mode=0, **over):
    gg, Y, eons, eonns, kw, rp, rx = C.owner_state(g, case, seed=seed, big=big)
    kw.update(over)
    mg.optimize_layout(Y, gg["head"], gg["tail"], gg["eps"], eons, eonns, n_threads=1, parallel=1, rev_indptr=rp,
                       rev_indices=rx, stream_mode=stream_mode, **kw)
    return gg, Y, eons, eonns, kw


def check_digests(own, case, arrays):
    for entry in own[f"digests_{case}"]:
        k, h = str(entry).split(":")
        assert C.digest(arrays[k]) == h, k


@pytest.mark.parametrize("case", EXACT)
def test_owner_bit_exact_against_reference(mg, golden, big_graph, case):
    g, own = golden("sgd_small.npz"), golden("sgd_owner.npz")
    _, Y, eons, eonns, kw = run_owner(mg, g, case, big_graph)
    assert np.array_equal(Y, own[f"Y_{case}"]), np.abs(Y - own[f"Y_{case}"]).max()
    check_digests(own, case, dict(eons=eons, eonns=eonns))


@pytest.mark.parametrize("case", CLOSE)
def test_owner_close_to_oracle_and_reference_quality(mg, golden, big_graph, case):
    g, own = golden("sgd_small.npz"), golden("sgd_owner.npz")
    # one epoch: the device and the oracle differ only by the last-place differences of powf / expf between CUDA
    # and the host libm, so positions agree to a few FP32 ulps of the layout's scale
    gg, Y1, _, _, kw1 = run_owner(mg, g, case, big_graph, epoch_end=1)
    _, Yo, eo, eno, kwo, rp, rx = C.owner_state(g, case, big=big_graph)
    kwo.update(epoch_end=1)
    O.sgd_owner(Yo, gg["head"], gg["tail"], gg["eps"], eo, eno, rev_indptr=rp, rev_indices=rx, **C.oracle_kw(kwo))
    assert np.abs(Y1 - Yo).max() <= 1e-5 * np.abs(Yo).max(), np.abs(Y1 - Yo).max()
    # forty epochs: the bookkeeping (and Adam's step counts) exactly as the reference's, the quality as its 8 seeds
    _, Y, eons, eonns, kw = run_owner(mg, g, case, big_graph)
    assert np.isfinite(Y).all()
    arrays = dict(eons=eons, eonns=eonns, adam_t=kw["adam_t"])
    for entry in own[f"digests_{case}"]:
        k, h = str(entry).split(":")
        if k in arrays:   # adam_m / adam_v carry the powf differences
            assert C.digest(arrays[k]) == h, k
    p_ref = own[f"purity_{case}"]
    p = np.mean([C.purity(run_owner(mg, g, case, big_graph, seed=sd)[1], gg["labels"]) for sd in range(1, 9)])
    assert p > p_ref.mean() - max(0.03, 1.5 * p_ref.std()), (p, p_ref.mean())


def test_owner_is_deterministic_and_ignores_stream_mode(mg, golden, big_graph):
    g = golden("sgd_small.npz")
    Ya = run_owner(mg, g, "gaussian_large", big_graph)[1]
    Yb = run_owner(mg, g, "gaussian_large", big_graph)[1]
    Yc = run_owner(mg, g, "gaussian_large", big_graph, stream_mode=1)[1]
    assert np.array_equal(Ya, Yb) and np.array_equal(Ya, Yc)


def test_owner_argument_errors(mg, golden, big_graph):
    g = golden("sgd_small.npz")
    gg, Y, eons, eonns, kw, rp, rx = C.owner_state(g, "b1_pairs", big=big_graph)
    head = gg["head"].copy()
    head[[10, 500]] = head[[500, 10]]
    with pytest.raises(RuntimeError, match="needs edges sorted by head"):
        mg.optimize_layout(Y, head, gg["tail"], gg["eps"], eons, eonns, n_threads=1, parallel=1, **kw)
    kw.update(loss=1)
    with pytest.raises(RuntimeError, match="supports the umap loss only"):
        mg.optimize_layout(Y, gg["head"], gg["tail"], gg["eps"], eons, eonns, n_threads=1, parallel=1, **kw)
    kw.update(loss=0, mid_rate=1e9)
    with pytest.raises(RuntimeError, match="mid_rate \\* row length / n_mid must be at most 65536"):
        mg.optimize_layout(Y, gg["head"], gg["tail"], gg["eps"], eons, eonns, n_threads=1, parallel=1,
                           rev_indptr=rp, rev_indices=rx, **kw)
    assert np.array_equal(Y, C.owner_state(g, "b1_pairs", big=big_graph)[1])


def test_owner_driver_on_blobs(mg):
    """the reference's owner-mode test (tests/test_magnet.py:387-401) through the package's SGD driver: a 3000-point
    6-blob kNN graph, 40 epochs with graph walks; two runs agree bit for bit and a 10-NN classifier on the layout
    scores above 0.95; InfoNCE is refused"""
    from sklearn.datasets import make_blobs
    from sklearn.neighbors import KNeighborsClassifier, kneighbors_graph
    from magnet_b200 import graph as G
    X, y = make_blobs(n_samples=3000, centers=6, n_features=20, random_state=0)
    A = kneighbors_graph(X.astype(np.float32), 15, mode="distance", include_self=False)
    A.data = np.exp(-A.data / A.data.mean()).astype(np.float32)
    A = ((A + A.T) * 0.5).tocsr()
    head, tail, eps = mg.edge_schedule(A, 40)
    a, b = mg.find_ab_params(1.0, 0.1)
    Y0 = G.initial_layout(G.pca2(X, 0), 0)
    outs = []
    for _ in range(2):
        Y = Y0.copy()
        mg.optimize_sgd(Y, head, tail, eps, 40, a=a, b=b, mid_weight=0.1, graph=A, seed=0, parallel="owner")
        outs.append(Y)
    assert np.array_equal(outs[0], outs[1])
    assert np.isfinite(outs[0]).all() and outs[0].shape == (3000, 2)
    assert KNeighborsClassifier(10).fit(outs[0], y).score(outs[0], y) > 0.95
    with pytest.raises(ValueError):
        mg.optimize_sgd(Y0.copy(), head, tail, eps, 40, a=a, b=b, loss=1, parallel="owner")
