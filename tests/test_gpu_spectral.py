"""The spectral initialisation's solver on the device (chebyshev_eigenvectors, src/spectral.cpp:141-241, as
magnet/spectral.py:8-46 calls it) against the reference's own compiled solver on the same graph and start block:
the leading n_wanted Ritz vectors span the same subspace (largest principal-angle sine below 1e-3), their Ritz
values agree to 1e-6, and the layout that spectral_init makes of them (the vectors scaled by 1 / sqrt(degree))
matches up to the orientation of each axis. Cases: the 10,000-point graph of the loss="umap" configuration (the
reference's own fuzzy graph), a graph of three connected components plus isolated nodes (per-component
deflation, zero degrees), and a 3-d layout (six columns)."""
import os
import sys

import numpy as np
import pytest
import scipy.sparse as sp

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
from spectral_cases import inputs, ritz_values, subspace_sine, three_components  # noqa: E402

pytestmark = pytest.mark.gpu


def compare(mg, ref, P, n_components, seed=0):
    from magnet_b200 import _native as N
    a = inputs(P, n_components, seed)
    Xd = N.chebyshev_eigenvectors(*a[:3], a[3].copy(), *a[4:], -1)
    Xr = np.asarray(ref.chebyshev_eigenvectors(*a[:3], a[3].copy(), *a[4:], -1))
    nw = n_components
    s = subspace_sine(Xd[:, :nw], Xr[:, :nw])
    vd, vr = ritz_values(sp.csr_matrix(P), a[4], Xd[:, :nw]), ritz_values(sp.csr_matrix(P), a[4], Xr[:, :nw])
    # the layout spectral_init makes: the vectors scaled by 1 / sqrt(degree), each axis up to its sign
    Ld, Lr = Xd[:, :nw] * a[4][:, None], Xr[:, :nw] * a[4][:, None]
    axes = [min(np.linalg.norm(Ld[:, c] - Lr[:, c]), np.linalg.norm(Ld[:, c] + Lr[:, c])) /
            max(np.linalg.norm(Lr[:, c]), 1e-30) for c in range(nw)]
    print("n=%d p=%d: principal-angle sine %.2e, Ritz values %s / %s, axis errors %s"
          % (P.shape[0], a[3].shape[1], s, np.round(vd, 7), np.round(vr, 7), np.round(axes, 6)))
    assert np.isfinite(Xd).all()
    assert s < 1e-3
    assert np.allclose(vd, vr, rtol=0, atol=1e-6)
    return axes


def test_umap_configuration_graph(mg, ref, golden):
    if ref is None:
        pytest.skip("reference module not built")
    g = golden("layout_config1.npz")
    P = sp.csr_matrix((g["data"], g["indices"], g["indptr"]), shape=(len(g["indptr"]) - 1,) * 2)
    axes = compare(mg, ref, P, 2)
    assert max(axes) < 1e-2


def test_components_and_isolated_nodes(mg, ref):
    if ref is None:
        pytest.skip("reference module not built")
    compare(mg, ref, three_components(), 2, seed=1)


def test_three_dimensions(mg, ref, golden):
    if ref is None:
        pytest.skip("reference module not built")
    g = golden("layout_config1.npz")
    P = sp.csr_matrix((g["data"], g["indices"], g["indptr"]), shape=(len(g["indptr"]) - 1,) * 2)
    compare(mg, ref, P, 3, seed=2)


def test_device_arrays_in_place(mg):
    import torch
    from magnet_b200 import _native as N
    a = inputs(three_components(), 2, seed=3)
    t = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()
    Xd = t(a[3])
    out = N.chebyshev_eigenvectors(t(a[0]), t(a[1]), t(a[2]), Xd, t(a[4]), t(a[5]), *a[6:], -1)
    assert out is Xd or out.data_ptr() == Xd.data_ptr()
    Xh = N.chebyshev_eigenvectors(*a[:3], a[3].copy(), *a[4:], -1)
    assert subspace_sine(Xd.cpu().numpy()[:, :2], Xh[:, :2]) < 1e-6


def test_wide_blocks_rejected(mg):
    from magnet_b200 import _native as N
    a = list(inputs(three_components(), 2))
    a[3] = np.zeros((a[3].shape[0], 9), np.float32)
    with pytest.raises(RuntimeError, match="at most 8 columns"):
        N.chebyshev_eigenvectors(*a, -1)


def test_one_wanted_vector_and_no_iterations(mg, ref, golden):
    """n_wanted = 1 (a three-column block), and max_iter = 0 (the start block's Rayleigh-Ritz only)"""
    if ref is None:
        pytest.skip("reference module not built")
    from magnet_b200 import _native as N
    g = golden("layout_config1.npz")
    P = sp.csr_matrix((g["data"], g["indices"], g["indptr"]), shape=(len(g["indptr"]) - 1,) * 2)
    compare(mg, ref, P, 1, seed=5)
    a = list(inputs(P, 2, seed=6))
    a[8] = 0
    Xd = N.chebyshev_eigenvectors(*a[:3], a[3].copy(), *a[4:], -1)
    Xr = np.asarray(ref.chebyshev_eigenvectors(*a[:3], a[3].copy(), *a[4:], -1))
    assert subspace_sine(Xd[:, :2], Xr[:, :2]) < 1e-6
