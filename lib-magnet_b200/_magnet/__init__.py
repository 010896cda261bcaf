"""Drop-in replacement of the reference's native module `_magnet` (kerighan/lib-magnet, src/bindings.cpp).

Put the directory holding this package ahead of the reference's extension on sys.path; the reference's Python
package (`magnet`) then runs its layout pass on the B200: optimize_layout, FFTConv2D, tsne_attraction, tsne_step,
tsne_update, bbox_2d, mid_spring, smooth_knn, mid_near_pairs_dense, knn_search and chebyshev_eigenvectors (blocks of
up to 8 columns) come from the device library. The host-side kernels that stay on the reference's code
(nn_descent, the sparse-data searches, subspace_iteration, louvain)
are forwarded to the reference's own compiled module, found through the MAGNET_HOST_MODULE environment variable
(path to the reference's `_magnet*.so`); without it they raise ImportError when used, as a missing `_magnet` would.
"""
import importlib.util as _ilu
import os as _os
import sys as _sys

from magnet_b200._native import (FFTConv2D, optimize_layout, tsne_attraction, tsne_step, tsne_update,  # noqa: F401
                                 bbox_2d, mid_spring, smooth_knn, mid_near_pairs_dense, knn_search)

_HOST_NAMES = ("nn_descent", "nn_descent_sparse", "knn_search_sparse", "mid_near_pairs_sparse", "subspace_iteration",
               "louvain", "interp_scatter",
               "interp_gather", "scatter_padded_2d", "spectral_products", "gather_forces_2d", "umap_attraction")


def _load_host():
    path = _os.environ.get("MAGNET_HOST_MODULE")
    if not path:
        return None
    # a module already loaded from the same file is reused: initialising a pybind11 extension twice in one
    # process registers its types twice
    for m in list(_sys.modules.values()):
        f = getattr(m, "__file__", None)
        if f and _os.path.realpath(f) == _os.path.realpath(path):
            return m
    spec = _ilu.spec_from_file_location("magnet_host_native._magnet", path)
    mod = _ilu.module_from_spec(spec)
    spec.loader.exec_module(mod)
    _sys.modules[spec.name] = mod   # so that a later loader of the same file finds it
    return mod


_host = _load_host()


def chebyshev_eigenvectors(indptr, indices, data, X, inv_sqrt_deg, component, n_wanted, degree, max_iter, tol,
                           n_threads=-1):
    """src/spectral.cpp:141-241 on the device for blocks of up to 8 columns (magnet/spectral.py asks for
    n_components + max(2, n_components)); wider blocks go to the reference's host module"""
    from magnet_b200 import _native
    if getattr(X, "shape", (0, 0))[1] <= 8:
        return _native.chebyshev_eigenvectors(indptr, indices, data, X, inv_sqrt_deg, component, n_wanted, degree,
                                              max_iter, tol, n_threads)
    if _host is None:
        raise ImportError("_magnet.chebyshev_eigenvectors with more than 8 columns runs on the reference's host "
                          "module; set MAGNET_HOST_MODULE to its path")
    return _host.chebyshev_eigenvectors(indptr, indices, data, X, inv_sqrt_deg, component, n_wanted, degree,
                                        max_iter, tol, n_threads)


def __getattr__(name):
    if name in _HOST_NAMES:
        if _host is None:
            raise ImportError(f"_magnet.{name} runs on the reference's host module; set MAGNET_HOST_MODULE to its path")
        return getattr(_host, name)
    raise AttributeError(name)
