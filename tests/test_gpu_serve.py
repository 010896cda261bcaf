"""The served form on the device (magnet_b200.serve): a fitted layout resident in HBM, transform() requests of
uneven sizes and a fit request admitted while others run, each worker on its own CUDA stream. Each transform
result is the same alone (one slot, one request at a time) and in the mix (four slots, all requests in flight):
owner mode makes the SGD a function of the request's inputs alone, and the rest of a request (kNN, memberships,
schedule) runs on its own stream and buffers. New points land among the training points of their own blob."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def blobs(n, d, centers, seed):
    rng = np.random.default_rng(seed)
    C = rng.normal(0, 6, (centers, d))
    y = rng.integers(0, centers, n)
    return (C[y] + rng.normal(0, 1, (n, d))).astype(np.float32), y


@pytest.mark.parametrize("search", ["beam", "exact"])
def test_transform_same_alone_and_in_the_mix(mg, cuda, search):
    """with the query kNN by beam search over the training graph (the reference's transform) and by exact
    blocked matmul"""
    from sklearn.neighbors import KNeighborsClassifier
    from magnet_b200 import serve as S
    X, y = blobs(4600, 16, 8, seed=3)
    Xtr, ytr, Xq, yq = X[:4000], y[:4000], X[4000:], y[4000:]
    Ytr, P = S.fit_layout(Xtr, n_epochs=100, seed=0, return_graph=True)
    a, b = mg.find_ab_params(1.0, 0.1)
    layout = S.FittedLayout(Xtr, Ytr, a=a, b=b, transform_epochs=60, graph=P if search == "beam" else None)
    sizes = [1, 37, 200, 5, 90, 150, 64, 53]
    chunks = np.split(Xq, np.cumsum(sizes)[:-1])

    srv = S.device_server(layout, slots=1)
    alone = [srv.submit("transform", (c, 7), layout.request_bytes(len(c)), len(c)).result(timeout=300)
             for c in chunks]
    srv.close()

    srv = S.device_server(layout, slots=4)
    futs = [srv.submit("transform", (c, 7), layout.request_bytes(len(c)), len(c)) for c in chunks[:4]]
    fit = srv.submit("fit", X[:3000], S.fit_bytes(3000, 16), 3000)
    futs += [srv.submit("transform", (c, 7), layout.request_bytes(len(c)), len(c)) for c in chunks[4:]]
    mixed = [f.result(timeout=300) for f in futs]
    Yfit = fit.result(timeout=300)
    srv.close()

    for c, ya, ym in zip(chunks, alone, mixed):
        assert ya.shape == (len(c), 2) and np.isfinite(ya).all()
        assert np.array_equal(ya, ym)
    assert Yfit.shape == (3000, 2) and np.isfinite(Yfit).all()
    clf = KNeighborsClassifier(10).fit(Ytr, ytr)
    assert clf.score(np.vstack(mixed), yq) > 0.9
    s = S.latency_summary(srv.done, "transform")
    assert s["requests"] == len(chunks) and s["points_per_s"] > 0
