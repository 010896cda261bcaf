"""Final-layout parity on the 10,000-point workload of the loss="umap" benchmark configuration (ten Gaussians in
d = 50, seed 0): the device's layouts against the reference's own on the same fuzzy graph P, initial layout Y0,
mid-near partners and kernel parameters, all captured from the reference's fit (tests/golden/make_layout_golden.py,
which also holds the reference's results). The bound is the layout pass's parity criterion: 15-NN preservation
(benchmarks/metrics.py:52-62) within +-0.005 and KL divergence within 1 %. Seeded layouts are compared on the mean
over the same 8 seeds (the reference's own runs scatter by 0.001-0.002 in 15-NN from one seed to the next; the
device's counter-mode draws are not the reference's stream, so single runs are not comparable).

Measured on B200 (mean over 8 seeds, device / reference):
  * umap, hogwild counter mode: printed by the test;
  * umap, serial stream mode: printed by the test;
  * hybrid: printed by the test;
  * tsne (one run): printed by the test.
"""
import os
import sys

import numpy as np
import pytest
import scipy.sparse as sp

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
import quality  # noqa: E402

pytestmark = pytest.mark.gpu

N, D, CENTRES, SEEDS = 10_000, 50, 10, 8


def config1_data(seed=0):
    """the benchmark's 10,000 x 50 data: centres N(0, 5^2 I), labels uniform, unit noise, default_rng(0)"""
    rng = np.random.default_rng(seed)
    C = rng.normal(0, 5.0, (CENTRES, D))
    y = rng.integers(0, CENTRES, N)
    return (C[y] + rng.normal(0, 1, (N, D))).astype(np.float32), y


@pytest.fixture(scope="module")
def case(golden):
    g = golden("layout_config1.npz")
    X, _ = config1_data()
    P = sp.csr_matrix((g["data"], g["indices"], g["indptr"]), shape=(N, N))
    P.has_sorted_indices = True
    return dict(g=g, X=X, P=P, hnn=quality.high_dim_neighbors(X))


def scores(case, Ys):
    k = [quality.knn_preservation(case["X"], Y, hnn=case["hnn"]) for Y in Ys]
    kl = [quality.kl_divergence(case["P"], Y) for Y in Ys]
    return float(np.mean(k)), float(np.mean(kl))


def check(case, name, Ys, ref_prefix):
    g = case["g"]
    assert all(np.isfinite(Y).all() for Y in Ys)
    k_d, kl_d = scores(case, Ys)
    k_r, kl_r = float(g["knn15_" + ref_prefix].mean()), float(g["kl_" + ref_prefix].mean())
    print("%s: 15-NN device %.4f reference %.4f (diff %+.4f); KL device %.4f reference %.4f (%+.2f %%)"
          % (name, k_d, k_r, k_d - k_r, kl_d, kl_r, 100 * (kl_d - kl_r) / kl_r))
    assert abs(k_d - k_r) <= 0.005, (k_d, k_r)
    assert abs(kl_d - kl_r) / kl_r <= 0.01, (kl_d, kl_r)


def sgd_layouts(mg, case, mid_w, **kw):
    g, P = case["g"], case["P"]
    head, tail, eps = mg.edge_schedule(P, int(g["n_epochs"]))
    out = []
    for j in range(SEEDS):
        Y = g["Y0"].copy()
        mg.optimize_sgd(Y, head, tail, eps, int(g["n_epochs"]), a=float(g["a"]), b=float(g["b"]),
                        rep_a=float(g["rep_a"]), rep_b=float(g["rep_b"]), mid_weight=mid_w,
                        mid_pairs=g["mid_pairs"], graph=P, seed=int(g["seed"]) + j, **kw)
        out.append(Y)
    return out


@pytest.mark.parametrize("mode", ["hogwild", "serial"])
def test_umap_layout_parity(mg, case, mode):
    """loss="umap", 500 epochs, against the reference at n_threads = 1: the counter mode (hogwild, the fast path)
    and the serial stream mode (the reference's single stream, replayed)"""
    Ys = sgd_layouts(mg, case, float(case["g"]["mid_w"]), parallel=mode)
    check(case, "umap " + mode, Ys, "umap")


def test_hybrid_layout_parity(mg, case):
    """loss="hybrid": the SGD pass with mid weight 0.2, the rescale and 300 full-batch iterations"""
    g, P = case["g"], case["P"]
    Ys = []
    for j in range(SEEDS):
        Ys.append(mg.hybrid_layout(P, g["Y0"].copy(), a=float(g["a"]), b=float(g["b"]), rep_a=float(g["rep_a"]),
                                   rep_b=float(g["rep_b"]), n_epochs=int(g["n_epochs"]), mid_pairs=g["mid_pairs"],
                                   mid_weight=0.2, seed=int(g["seed"]) + j, hybrid_iter=300))
    check(case, "hybrid", Ys, "hybrid")


def test_tsne_layout_parity(mg, case):
    """loss="tsne": 750 iterations with 250 of early exaggeration 12, from Y0 scaled to std 1e-4"""
    g = case["g"]
    Y = mg.optimize_tsne(case["P"], g["Y0_tsne"].copy(), n_iter=750, early_iter=250)
    check(case, "tsne", [Y], "tsne")
