"""The transform's edge schedule on the device (mg_transform_schedule; MAGNET.transform, magnet/__init__.py:907-912,
with _sampling_frequencies of magnet/__init__.py:51-66) against the host restatement that is pinned to the
reference's Python (`magnet_b200.drivers.sampling_frequencies`): the same kept edges in the same order, with eps
equal to the host's in float32 (the device solves s in FP64 by bisection and then exactly on its segment, the host
by a sorted cumulative sum, so a rounding difference of one FP64 ulp in s may move an eps by one float32 ulp)."""
import ctypes
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "lib-magnet_b200", "libmagnet_b200.so")


def schedule_device(w, ind, n_train, samples_per_node, n_epochs):
    import torch
    lib = ctypes.CDLL(LIB)
    P, I64 = ctypes.c_void_p, ctypes.c_int64
    lib.mg_transform_schedule.argtypes = [P, P, I64, ctypes.c_int, I64, ctypes.c_double, ctypes.c_int, P, P, P,
                                          ctypes.POINTER(I64)]
    lib.mg_last_error.restype = ctypes.c_char_p
    m, k = w.shape
    wd = torch.from_numpy(np.ascontiguousarray(w, dtype=np.float32)).cuda()
    idd = torch.from_numpy(np.ascontiguousarray(ind, dtype=np.int64)).cuda()
    head = torch.empty(m * k, dtype=torch.int32, device="cuda")
    tail = torch.empty(m * k, dtype=torch.int32, device="cuda")
    eps = torch.empty(m * k, dtype=torch.float32, device="cuda")
    kept = I64(0)
    rc = lib.mg_transform_schedule(P(wd.data_ptr()), P(idd.data_ptr()), m, k, n_train, samples_per_node, n_epochs,
                                   P(head.data_ptr()), P(tail.data_ptr()), P(eps.data_ptr()), ctypes.byref(kept))
    assert rc == 0, lib.mg_last_error()
    n = kept.value
    return head[:n].cpu().numpy(), tail[:n].cpu().numpy(), eps[:n].cpu().numpy()


def schedule_host(w, ind, n_train, samples_per_node, n_epochs):
    from magnet_b200 import drivers as D
    m, k = w.shape
    freq = D.sampling_frequencies(w.ravel().astype(np.float64), samples_per_node * m)
    keep = freq >= 1.0 / n_epochs
    head = (n_train + np.repeat(np.arange(m), k)).astype(np.int32)[keep]
    tail = ind.ravel().astype(np.int32)[keep]
    return head, tail, (1.0 / freq[keep]).astype(np.float32)


def memberships(m, k, seed, zeros=0.0):
    rng = np.random.default_rng(seed)
    w = np.sort(rng.random((m, k)).astype(np.float32) ** 3, axis=1)[:, ::-1]
    w[:, 0] = 1.0                                  # smooth_knn's first membership
    if zeros:
        w[rng.random((m, k)) < zeros] = 0.0
    return np.ascontiguousarray(w), rng.integers(0, 200000, (m, k))


@pytest.mark.parametrize("m,k,epochs,zeros", [(2048, 14, 100, 0.0), (1, 14, 100, 0.0), (37, 14, 200, 0.0),
                                              (4096, 14, 100, 0.3), (500, 29, 50, 0.0), (300, 14, 100, 0.95),
                                              (10, 4, 100, 0.2)])
def test_schedule_matches_host(mg, m, k, epochs, zeros):
    w, ind = memberships(m, k, seed=m + k, zeros=zeros)
    hd, td, ed = schedule_device(w, ind, 200000, 5.0, epochs)
    hh, th, eh = schedule_host(w, ind, 200000, 5.0, epochs)
    assert np.array_equal(hd, hh) and np.array_equal(td, th)
    rel = np.abs(ed.astype(np.float64) - eh) / eh
    assert rel.max() <= 1.2e-7 and np.mean(ed == eh) > 0.999, (rel.max(), np.mean(ed == eh))


def test_schedule_same_bits_every_call(mg):
    w, ind = memberships(1500, 14, seed=5)
    a = schedule_device(w, ind, 1000, 5.0, 100)
    b = schedule_device(w, ind, 1000, 5.0, 100)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))


def random_graph(n, deg, seed, zeros=0.0):
    import scipy.sparse as sp
    rng = np.random.default_rng(seed)
    rows = np.repeat(np.arange(n), deg)
    cols = rng.integers(0, n, n * deg)
    vals = (rng.random(n * deg) ** 3).astype(np.float32)
    if zeros:
        vals[rng.random(n * deg) < zeros] = 0.0
    P = sp.csr_matrix((vals, (rows, cols)), shape=(n, n))
    P.sum_duplicates()
    return P


@pytest.mark.parametrize("case", ["umap10k", "random", "zeros", "dense_target"])
def test_fit_schedule_matches_host(mg, golden, case):
    """MAGNET._edge_schedule (magnet/__init__.py:726-737) on the device against the host restatement pinned to the
    reference's Python: the same kept entries in CSR order, eps equal in float32 up to one ulp"""
    import scipy.sparse as sp
    from magnet_b200 import drivers as D
    if case == "umap10k":
        g = golden("layout_config1.npz")
        P = sp.csr_matrix((g["data"], g["indices"], g["indptr"]), shape=(len(g["indptr"]) - 1,) * 2)
        epochs, spn = 500, 5.0
    elif case == "random":
        P, epochs, spn = random_graph(20000, 15, 1), 200, 5.0
    elif case == "zeros":
        P, epochs, spn = random_graph(5000, 12, 2, zeros=0.6), 200, 5.0
    else:                                   # nnz <= samples_per_node * n: every frequency 1
        P, epochs, spn = random_graph(3000, 4, 3), 200, 5.0
    hh, th, eh = D.edge_schedule(P, epochs, spn)
    hd, td, ed = D.edge_schedule(P, epochs, spn, device=True)
    assert np.array_equal(hd, hh) and np.array_equal(td, th)
    rel = np.abs(ed.astype(np.float64) - eh) / eh
    assert rel.max() <= 1.2e-7 and np.mean(ed == eh) > 0.999, (rel.max(), np.mean(ed == eh))
