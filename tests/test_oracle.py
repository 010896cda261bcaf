"""The oracle (C restatement of the reference's layout pass) against the golden vectors the reference itself
produced (tests/golden/make_golden.py): bit-exact for the SGD at n_threads=1 and the t-SNE kernels."""
import numpy as np
import pytest

from oracle import oracle as O


def test_rng_stream_is_xorshift64star():
    # splitmix64 seeding + xorshift64* (src/rng.hpp:5-28), recomputed in Python integers
    seed = 12345
    z = (seed + 0x9E3779B97F4A7C15) & (2 ** 64 - 1)
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & (2 ** 64 - 1)
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & (2 ** 64 - 1)
    s = (z ^ (z >> 31)) | 1
    expect = []
    for _ in range(8):
        s ^= s >> 12
        s ^= (s << 25) & (2 ** 64 - 1)
        s ^= s >> 27
        expect.append((s * 0x2545F4914F6CDD1D) & (2 ** 64 - 1))
    assert [int(v) for v in O.rng_stream(seed, 8)] == expect


@pytest.mark.parametrize("case", ["default", "b1", "walk"])
def test_sgd_serial_bit_exact(golden, case):
    g = golden("sgd_small.npz")
    Y = g["Y0"].copy(); eps = g["eps"]; eons = eps.copy(); eonns = (eps / 5).astype(np.float32)
    kw = dict(a=1.7, b=0.8 if case != "b1" else 1.0, rep_a=1.7382, rep_b=1.0, seed=12345, epoch_start=0,
              epoch_end=40, alpha0=1.0, alpha1=0.0)
    if case == "default":
        kw.update(mid_pairs=g["mid_pairs"], mid_w0=0.1, mid_w1=0.0)
    if case == "walk":
        kw.update(indptr=g["indptr"], indices=g["indices"], mid_w0=0.1, mid_w1=0.0)
    O.sgd_serial(Y, g["head"], g["tail"], eps, eons, eonns, **kw)
    assert np.array_equal(Y, g[f"Y_{case}"])
    assert np.array_equal(eons, g[f"eons_{case}"]) and np.array_equal(eonns, g[f"eonns_{case}"])


def test_tsne_kernels_bit_exact(golden):
    g = golden("tsne_small.npz")
    import scipy.sparse as sp
    P = sp.csr_matrix((g["data"], g["indices"], g["indptr"]))
    Pn = P / P.sum()
    Pn = sp.csr_matrix(Pn, dtype=np.float32)
    a = O.tsne_attraction(Pn.indptr, Pn.indices, Pn.data, g["Yl"], 1.0)
    assert np.array_equal(a, g["attr"])
    assert np.array_equal(O.tsne_attraction(Pn.indptr, Pn.indices, Pn.data, g["Yl"], 0.7), g["attr07"])
    assert np.array_equal(np.array(O.bbox_2d(g["Yl"]), np.float32), g["bbox"])
    Y, U, G = g["Yl"].copy(), g["U"].copy(), g["G"].copy()
    O.tsne_step(Y, U, G, g["attr"], g["Fr"], 12.0, 1e-3, 250.0, 0.5)
    assert np.array_equal(U, g["Us"]) and np.array_equal(G, g["Gs"]) and np.array_equal(Y, g["Ys"])


def test_tsne_driver_restatement(golden):
    g = golden("tsne_small.npz")
    import scipy.sparse as sp
    P = sp.csr_matrix((g["data"], g["indices"], g["indptr"]))
    if O.reference() is None:
        pytest.skip("reference module not built")
    Y = O.optimize_tsne(P, g["Y0"].copy(), n_iter=60, early_iter=20, n_threads=1, backend="reference")
    assert np.array_equal(Y, g["Y_tsne60"])


@pytest.mark.parametrize("ni", [5, 3])
def test_grid_and_spectra_restatement(golden, ni):
    g = golden("fft_small.npz")
    xmin, ymin, width, nb = O.grid(g["Y"])
    assert np.allclose([xmin, ymin, width, nb], g[f"grid_{ni}"], rtol=0, atol=0)
    M, K1, K2 = O.kernel_spectra(nb, width, ni)
    assert M == int(g[f"M_{ni}"])
    assert np.array_equal([np.float64(K1).sum(), np.abs(np.float64(K1)).max()], g[f"K1h_sum_{ni}"])
    assert np.array_equal([np.float64(K2).sum(), np.abs(np.float64(K2)).max()], g[f"K2h_sum_{ni}"])


@pytest.mark.parametrize("ni", [5, 3])
def test_fft_fp64_oracle_against_reference(golden, ni):
    g = golden("fft_small.npz")
    xmin, ymin, width, nb = g[f"grid_{ni}"]
    sq, F = O.fft_repulsion_fp64(g["Y"], float(xmin), float(ymin), float(width), int(nb), ni)
    # the reference's FP32 FFT against the same interpolation with an exact convolution
    assert abs(sq - g[f"sumQ_{ni}"]) / g[f"sumQ_{ni}"] < 1e-5
    assert np.linalg.norm(F - g[f"F_{ni}"]) / np.linalg.norm(F) < 1e-4
    # and the interpolation against the exact all-pairs sums (the reference's own bounds, test_magnet.py:230-231)
    assert abs(sq - g["sumQ_exact"]) / g["sumQ_exact"] < 1e-3
    assert np.linalg.norm(F - g["F_exact"]) / np.linalg.norm(g["F_exact"]) < 2e-2


def test_exact_repulsion_oracle(golden):
    g = golden("fft_small.npz")
    sq, F = O.exact_repulsion(g["Y"])
    assert abs(sq - g["sumQ_exact"]) / g["sumQ_exact"] < 1e-12
    assert np.allclose(F, g["F_exact"], rtol=1e-9, atol=1e-12)


def test_schedule_record_matches_serial_run(golden):
    """the recorded draws are the ones the serial run consumes: replaying the schedule epoch by epoch advances
    eons / eonns exactly as the full run (the full run is bit-exact against the reference)"""
    g = golden("sgd_small.npz")
    eps = g["eps"]; eons = eps.copy(); eonns = (eps / 5).astype(np.float32)
    kw = dict(a=1.7, b=0.8, rep_a=1.7382, seed=12345, epoch_start=0, epoch_end=40, alpha0=1.0, alpha1=0.0,
              mid_pairs=g["mid_pairs"], mid_w0=0.1, mid_w1=0.0)
    for e in range(40):
        sampled, n_neg, off, negs, mid = O.sgd_schedule(g["Y0"].copy(), g["head"], g["tail"], eps, eons, eonns, e, **kw)
        assert negs.size == n_neg.sum()
        assert ((negs >= 0) & (negs < g["Y0"].shape[0])).all()
    assert np.array_equal(eons, g["eons_default"]) and np.array_equal(eonns, g["eonns_default"])
