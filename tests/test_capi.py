"""The C-ABI library loads and exports every entry point include/magnet_b200.h declares; the pybind11 surface
keeps the reference's names (no compute call: these run without a GPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "magnet_b200.h")
LIB = os.path.join(ROOT, "lib-magnet_b200", "libmagnet_b200.so")


def declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mg_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_entry_points():
    names = declared()
    for must in ("mg_fftconv_create", "mg_fftconv_compute", "mg_optimize_layout", "mg_optimize_tsne",
                 "mg_tsne_attraction", "mg_tsne_step", "mg_bbox_2d", "mg_last_error", "mg_smooth_knn",
                 "mg_fuzzy_union"):
        assert must in names


def test_library_exports_every_declared_symbol():
    if not os.path.exists(LIB):
        pytest.skip("library not built (run __graft_entry__.build())")
    lib = ctypes.CDLL(LIB)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_error_convention_without_gpu():
    if not os.path.exists(LIB):
        pytest.skip("library not built")
    lib = ctypes.CDLL(LIB)
    lib.mg_last_error.restype = ctypes.c_char_p
    h = ctypes.c_void_p()
    # argument errors are raised before any device work: M must be 5-smooth
    rc = lib.mg_fftconv_create(7 * 11, 3, ctypes.byref(h))
    assert rc == 1 and b"5-smooth" in lib.mg_last_error()


def test_graph_argument_errors_without_gpu():
    if not os.path.exists(LIB):
        pytest.skip("library not built")
    lib = ctypes.CDLL(LIB)
    lib.mg_last_error.restype = ctypes.c_char_p
    P, I64 = ctypes.c_void_p, ctypes.c_int64
    lib.mg_fuzzy_union.argtypes = [P, P, I64, ctypes.c_int, I64, ctypes.c_double, P, P, P, I64, ctypes.POINTER(I64)]
    lib.mg_smooth_knn.argtypes = [P, I64, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_int, P]
    nnz = I64(0)
    buf = (ctypes.c_int32 * 8)()
    # a graph of 4 nodes cannot hold 6 kNN rows
    rc = lib.mg_fuzzy_union(buf, buf, 6, 1, 4, 1.0, buf, buf, buf, 8, ctypes.byref(nnz))
    assert rc == 1 and b"n_rows <= n" in lib.mg_last_error()
    rc = lib.mg_smooth_knn(buf, 2, 2, 0, 1.0, 64, buf)
    assert rc == 1 and b"n_neighbors must be positive" in lib.mg_last_error()


def test_native_surface_has_reference_names():
    mod = pytest.importorskip("magnet_b200._native")
    for name in ("FFTConv2D", "optimize_layout", "tsne_attraction", "tsne_step", "tsne_update", "bbox_2d",
                 "mid_spring", "smooth_knn", "fuzzy_union"):
        assert hasattr(mod, name)
    import _magnet
    assert _magnet.optimize_layout is mod.optimize_layout
    assert _magnet.smooth_knn is mod.smooth_knn


def test_owner_mode_argument_rules_without_gpu(golden):
    """owner mode's argument rules (src/layout.cpp:375-377, 441-446) and the reverse-pull bound are checked on
    the host before any device work"""
    pytest.importorskip("magnet_b200._native")
    import numpy as np
    import magnet_b200 as mg
    import sgd_cases as C
    g = golden("sgd_small.npz")
    gg, Y, eons, eonns, kw, rp, rx = C.owner_state(g, "b1_pairs")
    args = (Y, gg["head"], gg["tail"], gg["eps"], eons, eonns)
    with pytest.raises(RuntimeError, match="supports the umap loss only"):
        mg.optimize_layout(*args, n_threads=1, parallel=1, **(kw | dict(loss=1)))
    head = gg["head"].copy()
    head[[10, 500]] = head[[500, 10]]
    with pytest.raises(RuntimeError, match="needs edges sorted by head"):
        mg.optimize_layout(Y, head, *args[2:], n_threads=1, parallel=1, **kw)
    with pytest.raises(RuntimeError, match="at most 65536"):
        mg.optimize_layout(*args, n_threads=1, parallel=1, rev_indptr=rp, rev_indices=rx, **(kw | dict(mid_rate=1e9)))
    with pytest.raises(RuntimeError, match="owner_chunk_edges"):
        mg.optimize_layout(*args, n_threads=1, parallel=1, owner_chunk_edges=-1, **kw)
    assert np.array_equal(Y, C.owner_state(g, "b1_pairs")[1])


def test_transform_schedule_argument_errors_without_gpu():
    if not os.path.exists(LIB):
        pytest.skip("library not built")
    lib = ctypes.CDLL(LIB)
    lib.mg_last_error.restype = ctypes.c_char_p
    P, I64 = ctypes.c_void_p, ctypes.c_int64
    lib.mg_transform_schedule.argtypes = [P, P, I64, ctypes.c_int, I64, ctypes.c_double, ctypes.c_int, P, P, P,
                                          ctypes.POINTER(I64)]
    kept = I64(0)
    rc = lib.mg_transform_schedule(None, None, 4, 3, 10, 5.0, 0, None, None, None, ctypes.byref(kept))
    assert rc == 1 and b"n_epochs" in lib.mg_last_error()
    rc = lib.mg_transform_schedule(None, None, 4, 3, 10, 5.0, 100, None, None, None, None)
    assert rc == 1 and b"n_kept" in lib.mg_last_error()


def test_chebyshev_argument_errors_without_gpu():
    if not os.path.exists(LIB):
        pytest.skip("library not built")
    lib = ctypes.CDLL(LIB)
    lib.mg_last_error.restype = ctypes.c_char_p
    P, I64 = ctypes.c_void_p, ctypes.c_int64
    lib.mg_chebyshev_eigenvectors.argtypes = [P, P, P, I64, I64, P, ctypes.c_int, P, P, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_int, ctypes.c_float]
    import numpy as np
    X = np.zeros((4, 3), np.float32)
    rc = lib.mg_chebyshev_eigenvectors(None, None, None, 4, 0, X.ctypes.data, 3, None, None, 3, 30, 5, 0.05)
    assert rc == 1 and b"n_wanted + 1 columns" in lib.mg_last_error()
    rc = lib.mg_chebyshev_eigenvectors(None, None, None, 4, 0, X.ctypes.data, 3, None, None, 2, 1, 5, 0.05)
    assert rc == 1 and b"degree must be >= 2" in lib.mg_last_error()


def test_edge_schedule_argument_errors_without_gpu():
    if not os.path.exists(LIB):
        pytest.skip("library not built")
    lib = ctypes.CDLL(LIB)
    lib.mg_last_error.restype = ctypes.c_char_p
    P, I64 = ctypes.c_void_p, ctypes.c_int64
    lib.mg_edge_schedule.argtypes = [P, P, P, I64, I64, ctypes.c_double, ctypes.c_int, P, P, P, ctypes.POINTER(I64)]
    import numpy as np
    ip = np.array([0, 1, 2], np.int32)
    kept = I64(0)
    rc = lib.mg_edge_schedule(ip.ctypes.data, None, None, 2, 2, 5.0, 100, None, None, None, ctypes.byref(kept))
    assert rc == 1 and b"nnz entries" in lib.mg_last_error()
    rc = lib.mg_edge_schedule(ip.ctypes.data, None, None, 2, 0, 5.0, 0, None, None, None, ctypes.byref(kept))
    assert rc == 1 and b"n_epochs" in lib.mg_last_error()
