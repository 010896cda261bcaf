"""Generates tests/golden/layout_config1.npz: final layouts of the reference (kerighan/lib-magnet 3.0.2) on the
10,000-point workload of the loss="umap" benchmark configuration, for the final-layout parity tests.

Data: n = 10,000 points in d = 50, ten centres drawn N(0, 5^2 I), labels uniform, X = centre + N(0, I), from
numpy's default_rng(0) in that order (centres, labels, noise). The reference builds everything else with its own
code: MAGNET(loss="umap", n_epochs=500, n_threads=1, random_state=0).fit(X) gives the NN-descent fuzzy graph P,
its spectral initial layout Y0, its mid-near partners, (a, b) and the SGD seed; those are captured from its
optimize_layout call and stored. The reference's results on that (P, Y0):
  * umap: its optimize_layout at n_threads=1 (deterministic), for the fit's seed and 7 more;
  * hybrid: the loss="hybrid" sequence (magnet/__init__.py:683-700): SGD with mid weight 0.2, the rescale to
    std 31 sqrt(n / 70000), 300 full-batch iterations of magnet/tsne.py optimize_tsne, for 8 seeds (n_threads=1);
  * tsne: magnet/tsne.py optimize_tsne on (P, Y0 scaled to std 1e-4), 750 iterations with 250 of early
    exaggeration 12 (the loss="tsne" benchmark's schedule).
Each result is stored with its 15-NN preservation (benchmarks/metrics.py) and its KL divergence (quality.py).

Runs only where the reference checkout is available (MAGNET_REFERENCE_DIR, else the folder `reference` beside
this repository) and its native module has been compiled by oracle/build_ref.sh.

    python tests/golden/make_layout_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("MAGNET_REFERENCE_DIR", os.path.join(os.path.dirname(ROOT), "reference"))
sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))   # the compiled reference module, importable as _magnet
sys.path.insert(0, REF)
sys.path.insert(0, HERE)

import _magnet  # noqa: E402  (the reference's native module)
from magnet import MAGNET  # noqa: E402
from magnet.tsne import optimize_tsne  # noqa: E402
import quality  # noqa: E402

N, D, CENTRES = 10_000, 50, 10
SEEDS = 8


def config1_data(seed=0):
    rng = np.random.default_rng(seed)
    C = rng.normal(0, 5.0, (CENTRES, D))
    y = rng.integers(0, CENTRES, N)
    X = (C[y] + rng.normal(0, 1, (N, D))).astype(np.float32)
    return X, y


def capture_fit(X):
    """the reference's umap fit, with the arguments of its optimize_layout call recorded"""
    calls = []
    real = _magnet.optimize_layout

    def spy(*args):
        calls.append([np.array(a, copy=True) if isinstance(a, np.ndarray) else a for a in args])
        return real(*args)
    _magnet.optimize_layout = spy
    try:
        est = MAGNET(loss="umap", n_epochs=500, n_threads=1, random_state=0).fit(X)
    finally:
        _magnet.optimize_layout = real
    assert len(calls) == 1, len(calls)
    return est, calls[0]


def sgd_run(args, seed, mid_w=None, n_threads=1):
    """the captured optimize_layout call with another seed (and mid weight); returns Y"""
    a = [np.array(x, copy=True) if isinstance(x, np.ndarray) else x for x in args]
    if mid_w is not None:
        a[12], a[13] = float(mid_w), 0.0          # mid_w0, mid_w1: the single call's linear decay to 0
    a[39], a[40] = int(seed), int(n_threads)      # seed, n_threads
    _magnet.optimize_layout(*a)
    return a[0]


def main():
    X, y = config1_data()
    est, args = capture_fit(X)
    P = est.graph_.tocsr()
    P.sort_indices()
    Y0 = args[0]
    seed0 = int(args[39])
    hnn = quality.high_dim_neighbors(X)
    out = dict(indptr=P.indptr.astype(np.int32), indices=P.indices.astype(np.int32), data=P.data.astype(np.float32),
               Y0=Y0, mid_pairs=np.asarray(args[33], np.int32), a=np.float64(args[14]), b=np.float64(args[15]),
               rep_a=np.float64(args[16]), rep_b=np.float64(args[17]), seed=np.int64(seed0),
               mid_w=np.float64(args[12]), n_epochs=np.int64(args[9]))
    assert np.array_equal(est.embedding_, sgd_run(args, seed0)), "the captured call does not replay the fit"

    def stats(prefix, Ys):
        out["knn15_" + prefix] = np.array([quality.knn_preservation(X, Yk, hnn=hnn) for Yk in Ys])
        out["kl_" + prefix] = np.array([quality.kl_divergence(P, Yk) for Yk in Ys])
        out["Y_" + prefix] = Ys[0]
        print(prefix, "15-NN", out["knn15_" + prefix].round(4), "KL", out["kl_" + prefix].round(4), flush=True)

    seeds = [seed0 + j for j in range(SEEDS)]
    stats("umap", [sgd_run(args, s) for s in seeds])

    hyb = []
    for s in seeds:
        Yh = sgd_run(args, s, mid_w=0.2)
        Yh -= Yh.mean(0)
        Yh *= 31.0 * np.sqrt(N / 70000.0) / max(float(Yh[:, 0].std()), 1e-12)
        hyb.append(optimize_tsne(P, Yh, n_iter=300, early_iter=0, exaggeration=1.0, n_threads=1))
    stats("hybrid", hyb)

    Yt = (Y0 / max(float(Y0[:, 0].std()), 1e-12) * 1e-4).astype(np.float32)
    out["Y0_tsne"] = Yt.copy()
    stats("tsne", [optimize_tsne(P, Yt.copy(), n_iter=750, early_iter=250, n_threads=1)])
    np.savez_compressed(os.path.join(HERE, "layout_config1.npz"), **out)


if __name__ == "__main__":
    main()
