"""Mid-near partners on the device (mid_near_pairs_dense, src/nndescent.cpp:731-768) against the reference's own
compiled module and the oracle's C restatement: the same partners bit for bit for the same seed and thread count,
on the host's distance kernel and on the two others (MAGNET_DISTANCE_ORDER)."""
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def data(n, d, seed):
    rng = np.random.default_rng(seed)
    C = rng.normal(0, 4, (7, d))
    return (C[rng.integers(0, 7, n)] + rng.normal(0, 1, (n, d))).astype(np.float32)


@pytest.mark.parametrize("n,d,nt,seed", [(5000, 50, 1, 0), (9000, 50, 3, 11), (20000, 32, -1, 2), (6000, 10, 2, 5),
                                         (7, 1, 1, 3), (4096, 64, 64, 9), (100_000, 50, -1, 2)])
def test_mid_near_pairs_match_reference(mg, ref, n, d, nt, seed):
    X = data(n, d, seed)
    got = mg._native.mid_near_pairs_dense(X, 5, 6, seed, nt)
    assert got.shape == (n, 5) and got.dtype == np.int32
    if ref is not None:
        assert np.array_equal(got, np.asarray(ref.mid_near_pairs_dense(X, 5, 6, seed, nt)))
    assert np.array_equal(got, O.mid_near_pairs(X, 5, 6, seed, nt))


@pytest.mark.parametrize("order", [0, 1, 2])
def test_mid_near_pairs_distance_orders(mg, order, monkeypatch):
    """each of the reference's three squared-distance kernels, against the oracle's restatement of it"""
    X = data(12000, 37, 4)
    monkeypatch.setenv("MAGNET_DISTANCE_ORDER", str(order))
    got = mg._native.mid_near_pairs_dense(X, 4, 7, 21, 5)
    assert np.array_equal(got, O.mid_near_pairs(X, 4, 7, 21, 5, order=order))


def test_mid_near_pairs_device_arrays_and_rules(mg):
    import torch
    X = data(3000, 20, 1)
    Xd = torch.from_numpy(X).cuda()
    got = mg._native.mid_near_pairs_dense(Xd, 5, 6, 7, 2)
    assert np.array_equal(got, O.mid_near_pairs(X, 5, 6, 7, 2))
    with pytest.raises(RuntimeError, match="need n_pairs >= 1, n_cand >= 2 and n > n_cand"):
        mg._native.mid_near_pairs_dense(X[:6], 5, 6, 0, 1)
    with pytest.raises(RuntimeError, match="need n_pairs >= 1, n_cand >= 2 and n > n_cand"):
        mg._native.mid_near_pairs_dense(X, 5, 1, 0, 1)
