"""TEST ORACLE — not part of the product.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference legs import this module, and only
as the checker or as the timed CPU baseline. It gives:

* ``lib()``: the plain-C restatement ``magnet_oracle.c`` (ctypes), built by ``build()`` into oracle/_build/;
* ``reference()``: the reference's own native module compiled from its sources by ``build_ref.sh`` into
  oracle/_ref/ (present when the reference checkout was available at build time);
* numpy restatements of the reference's Python drivers for the layout pass:
  ``grid`` (magnet/tsne.py:30-46), ``kernel_spectra`` (magnet/tsne.py:48-71), ``optimize_tsne``
  (magnet/tsne.py:132-214, the common fused path), ``sampling_frequencies`` / ``edge_schedule``
  (magnet/__init__.py:51-66, 727-737) and ``optimize_sgd`` (MAGNET._optimize, magnet/__init__.py:751-839,
  integer-epoch path);
* ``fft_repulsion_fp64``: the FFT-interpolated repulsion with the reference's spread/gather and an FP64
  convolution, and ``exact_repulsion``: the FP64 all-pairs sums;
* ``chebyshev_eigenvectors``: a numpy restatement of the spectral init's solver (src/spectral.cpp:141-241).
"""
import ctypes
import importlib.util
import os
import subprocess
import sys
import glob

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_BUILD = os.path.join(HERE, "_build")
_LIB_PATH = os.path.join(_BUILD, "libmagnet_oracle.so")
_REF_DIR = os.path.join(HERE, "_ref")

_lib = None
_ref = None


def build(force=False):
    """Compile the C restatement (gcc, IEEE single ops, no FMA contraction)."""
    src = os.path.join(HERE, "magnet_oracle.c")
    if not force and os.path.exists(_LIB_PATH) and os.path.getmtime(_LIB_PATH) >= os.path.getmtime(src):
        return _LIB_PATH
    os.makedirs(_BUILD, exist_ok=True)
    tmp = _LIB_PATH + ".tmp"
    subprocess.check_call(["gcc", "-O2", "-fPIC", "-shared", "-std=c11", "-ffp-contract=off", "-fno-fast-math",
                           src, "-o", tmp, "-lm"])
    os.replace(tmp, _LIB_PATH)
    return _LIB_PATH


def build_reference():
    """Compile the reference's native module from its sources (oracle/build_ref.sh); no-op when up to date or
    when the sources are absent but a prebuilt module exists."""
    subprocess.check_call(["bash", os.path.join(HERE, "build_ref.sh")])


_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_F = ctypes.c_float


class SgdArgs(ctypes.Structure):
    _fields_ = [
        ("Y", _P), ("n", _I64), ("dim", ctypes.c_int),
        ("head", _P), ("tail", _P), ("eps", _P), ("eons", _P), ("eonns", _P), ("n_edges", _I64),
        ("indptr", _P), ("indices", _P), ("walk_lens", _P), ("mid_pairs", _P), ("n_mid", ctypes.c_int),
        ("jump_indptr", _P), ("jump_indices", _P), ("mid_jump", _F),
        ("epoch_start", ctypes.c_int), ("epoch_end", ctypes.c_int), ("alpha0", _F), ("alpha1", _F),
        ("mid_w0", _F), ("mid_w1", _F),
        ("a", _F), ("b", _F), ("rep_a", _F), ("rep_b", _F), ("negative_sample_rate", _F), ("loss", ctypes.c_int),
        ("exaggeration", _F), ("repulsion_strength", _F), ("walk_len", ctypes.c_int), ("mid_rate", _F),
        ("optimizer", ctypes.c_int), ("clip_mode", ctypes.c_int), ("n_fixed", _I64),
        ("adam_m", _P), ("adam_v", _P), ("adam_t", _P), ("beta1", _F), ("beta2", _F),
        ("kernel", ctypes.c_int), ("node_b", _P), ("seed", ctypes.c_uint64),
    ]


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        L.orc_rng_stream.argtypes = [ctypes.c_uint64, _I64, _P]
        L.orc_sgd_serial.argtypes = [ctypes.POINTER(SgdArgs), ctypes.c_int]
        L.orc_sgd_serial.restype = ctypes.c_int
        L.orc_sgd_owner.argtypes = [ctypes.POINTER(SgdArgs), _P, _P]
        L.orc_sgd_owner.restype = ctypes.c_int
        L.orc_owner_chunks.argtypes = [_P, _I64, _I64, _P, _P]
        L.orc_owner_chunks.restype = ctypes.c_int
        L.orc_smooth_knn.argtypes = [_P, _I64, ctypes.c_int, ctypes.c_int, _F, ctypes.c_int, _P]
        L.orc_fuzzy_union.argtypes = [_P, _P, _I64, ctypes.c_int, _I64, ctypes.c_double, _P, _P, _P, _I64]
        L.orc_fuzzy_union.restype = _I64
        L.orc_sgd_schedule.argtypes = [ctypes.POINTER(SgdArgs), ctypes.c_int, ctypes.c_int, _P, _P, _P, _P, _I64, _P]
        L.orc_sgd_schedule.restype = _I64
        L.orc_spread.argtypes = [_P, _I64, _F, _F, _F, ctypes.c_int, ctypes.c_int, _P]
        L.orc_gather.argtypes = [_P, _I64, _F, _F, _F, ctypes.c_int, ctypes.c_int, _P, _P]
        L.orc_gather.restype = ctypes.c_double
        L.orc_exact_repulsion.argtypes = [_P, _I64, _I64, _I64, ctypes.c_double, _P]
        L.orc_exact_repulsion.restype = ctypes.c_double
        L.orc_tsne_attraction.argtypes = [_P, _P, _P, _P, _I64, ctypes.c_int, _F, _P]
        L.orc_tsne_step.argtypes = [_P, _P, _P, _P, _P, _I64, ctypes.c_int, _F, _F, _F, _F]
        L.orc_bbox_2d.argtypes = [_P, _I64, _P]
        L.orc_mid_near_pairs.argtypes = [_P, _I64, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint64,
                                         ctypes.c_int, ctypes.c_int, _P]
        L.orc_mid_near_pairs.restype = ctypes.c_int
        _lib = L
    return _lib


def reference():
    """The reference's compiled module (oracle/_ref/_magnet*.so), loaded under a private name so that it never
    shadows a `_magnet` module of the product. None when it was not built."""
    global _ref
    if _ref is None:
        cands = glob.glob(os.path.join(_REF_DIR, "_magnet*.so"))
        if not cands:
            return None
        # a process that already imported the same file (e.g. as `_magnet` for the reference's Python package)
        # must reuse it: initialising the extension twice registers its pybind11 types twice
        for m in list(sys.modules.values()):
            f = getattr(m, "__file__", None)
            if f and os.path.realpath(f) == os.path.realpath(cands[0]):
                _ref = m
                return _ref
        spec = importlib.util.spec_from_file_location("magnet_reference_native._magnet", cands[0])
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        sys.modules[spec.name] = mod   # visible to other loaders of the same file in this process
        _ref = mod
    return _ref


def _ptr(a):
    return None if a is None else a.ctypes.data


def _c32(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


# ---------------------------------------------------------------------------------------------- RNG
def rng_stream(seed, count):
    out = np.empty(count, dtype=np.uint64)
    lib().orc_rng_stream(ctypes.c_uint64(seed & (2 ** 64 - 1)), count, out.ctypes.data)
    return out


# ---------------------------------------------------------------------------------------------- SGD
def _sgd_args(Y, head, tail, eps, eons, eonns, *, indptr=None, indices=None, walk_lens=None, mid_pairs=None,
              jump_indptr=None, jump_indices=None, mid_jump=0.0, epoch_start=0, epoch_end=1, alpha0=1.0,
              alpha1=1.0, mid_w0=0.0, mid_w1=0.0, a=1.577, b=0.895, rep_a=None, rep_b=1.0,
              negative_sample_rate=5.0, loss=0, exaggeration=1.0, repulsion_strength=2.0, walk_len=4,
              mid_rate=0.25, optimizer=0, clip_mode=0, n_fixed=0, adam_m=None, adam_v=None, adam_t=None,
              beta1=0.9, beta2=0.999, kernel=0, node_b=None, seed=0, keep=None):
    n, dim = Y.shape
    if rep_a is None:
        rep_a = a
    args = SgdArgs()
    args.Y = Y.ctypes.data; args.n = n; args.dim = dim
    args.head = head.ctypes.data; args.tail = tail.ctypes.data; args.eps = eps.ctypes.data
    args.eons = eons.ctypes.data; args.eonns = eonns.ctypes.data; args.n_edges = head.shape[0]
    args.indptr = _ptr(indptr); args.indices = _ptr(indices); args.walk_lens = _ptr(walk_lens)
    if mid_pairs is not None and mid_pairs.size > 0:
        args.mid_pairs = mid_pairs.ctypes.data; args.n_mid = mid_pairs.shape[1]
    else:
        args.mid_pairs = None; args.n_mid = 0
    if jump_indptr is not None and jump_indptr.size > 0:
        args.jump_indptr = jump_indptr.ctypes.data; args.jump_indices = jump_indices.ctypes.data
    args.mid_jump = mid_jump
    args.epoch_start = epoch_start; args.epoch_end = epoch_end
    args.alpha0 = alpha0; args.alpha1 = alpha1; args.mid_w0 = mid_w0; args.mid_w1 = mid_w1
    args.a = a; args.b = b; args.rep_a = rep_a; args.rep_b = rep_b
    args.negative_sample_rate = negative_sample_rate; args.loss = loss; args.exaggeration = exaggeration
    args.repulsion_strength = repulsion_strength; args.walk_len = walk_len; args.mid_rate = mid_rate
    args.optimizer = optimizer; args.clip_mode = clip_mode; args.n_fixed = n_fixed
    args.adam_m = _ptr(adam_m); args.adam_v = _ptr(adam_v); args.adam_t = _ptr(adam_t)
    args.beta1 = beta1; args.beta2 = beta2; args.kernel = kernel; args.node_b = _ptr(node_b)
    args.seed = ctypes.c_uint64(seed & (2 ** 64 - 1)).value
    return args


def sgd_serial(Y, head, tail, eps, eons, eonns, per_edge_stream=False, **kw):
    """optimize_layout at n_threads=1 (in place on Y, eons, eonns and the Adam state)."""
    for a in (Y, eons, eonns):
        assert a.flags.c_contiguous
    args = _sgd_args(Y, head, tail, eps, eons, eonns, **kw)
    lib().orc_sgd_serial(ctypes.byref(args), int(bool(per_edge_stream)))


def sgd_owner(Y, head, tail, eps, eons, eonns, rev_indptr=None, rev_indices=None, **kw):
    """optimize_layout with parallel=1 (owner mode), in place; the result does not depend on the thread count."""
    for a in (Y, eons, eonns):
        assert a.flags.c_contiguous
    args = _sgd_args(Y, head, tail, eps, eons, eonns, **kw)
    rp = None if rev_indptr is None or rev_indptr.size == 0 else _c32(rev_indptr, np.int32)
    rx = None if rp is None else _c32(rev_indices, np.int32)
    if lib().orc_sgd_owner(ctypes.byref(args), _ptr(rp), _ptr(rx)) != 0:
        raise ValueError("owner mode needs edges sorted by head and the umap loss")


def owner_chunks(head, n):
    """(own, eown): first node and first edge of each owner-mode chunk, n_chunks + 1 entries each"""
    head = _c32(head, np.int32)
    nc = lib().orc_owner_chunks(head.ctypes.data, head.shape[0], n, None, None)
    own = np.zeros(nc + 1, np.int64); eown = np.zeros(nc + 1, np.int64)
    lib().orc_owner_chunks(head.ctypes.data, head.shape[0], n, own.ctypes.data, eown.ctypes.data)
    return own, eown


def sgd_schedule(Y, head, tail, eps, eons, eonns, epoch, per_edge_stream=False, negs_cap=None, **kw):
    """Draws of one epoch: (sampled u8[E], n_neg i32[E], neg_off i64[E], negs i32[total], mid i32[E]).
    eons / eonns are advanced in place."""
    E = head.shape[0]
    sampled = np.zeros(E, np.uint8); n_neg = np.zeros(E, np.int32); neg_off = np.zeros(E, np.int64)
    mid = np.zeros(E, np.int32)
    cap = negs_cap if negs_cap is not None else int(E * (float(kw.get("negative_sample_rate", 5.0)) + 2) + 64)
    negs = np.zeros(cap, np.int32)
    args = _sgd_args(Y, head, tail, eps, eons, eonns, **kw)
    tot = lib().orc_sgd_schedule(ctypes.byref(args), int(epoch), int(bool(per_edge_stream)), sampled.ctypes.data,
                                 n_neg.ctypes.data, neg_off.ctypes.data, negs.ctypes.data, cap, mid.ctypes.data)
    assert tot <= cap, "negative buffer too small"
    return sampled, n_neg, neg_off, negs[:tot], mid


# ---------------------------------------------------------------------------------------------- fuzzy graph
def smooth_knn(dist, n_neighbors, bandwidth=1.0, n_iter=64):
    """src/graph.cpp:29-78 on one host thread: memberships (n, k) float32"""
    dist = _c32(dist, np.float32)
    n, k = dist.shape
    out = np.empty_like(dist)
    lib().orc_smooth_knn(dist.ctypes.data, n, k, int(n_neighbors), float(bandwidth), int(n_iter), out.ctypes.data)
    return out


def fuzzy_union(ind, vals, n=None, set_op_mix_ratio=1.0):
    """the union of magnet/knn.py:221-230 given the memberships: (indptr, indices, data) of the n x n CSR"""
    ind = _c32(ind, np.int32)
    vals = _c32(vals, np.float32)
    rows, k = ind.shape
    n = rows if n is None else int(n)
    cap = max(2 * rows * k, 1)
    indptr = np.zeros(n + 1, np.int32); indices = np.zeros(cap, np.int32); data = np.zeros(cap, np.float32)
    nnz = lib().orc_fuzzy_union(ind.ctypes.data, vals.ctypes.data, rows, k, n, float(set_op_mix_ratio),
                                indptr.ctypes.data, indices.ctypes.data, data.ctypes.data, cap)
    if nnz < 0:
        raise ValueError("neighbour index out of range")
    return indptr, indices[:nnz], data[:nnz]


# ---------------------------------------------------------------------------------------------- t-SNE kernels
def tsne_attraction(indptr, indices, data, Y, dof=1.0):
    n, dim = Y.shape
    out = np.empty_like(Y)
    lib().orc_tsne_attraction(_c32(indptr, np.int32).ctypes.data, _c32(indices, np.int32).ctypes.data,
                              _c32(data, np.float32).ctypes.data, Y.ctypes.data, n, dim, dof, out.ctypes.data)
    return out


def tsne_step(Y, U, G, A, F, rho, inv_sumQ, lr, momentum):
    n, dim = Y.shape
    lib().orc_tsne_step(Y.ctypes.data, U.ctypes.data, G.ctypes.data, _c32(A, np.float32).ctypes.data,
                        _c32(F, np.float32).ctypes.data, n, dim, rho, inv_sumQ, lr, momentum)


def bbox_2d(Y):
    out = np.empty(4, np.float32)
    lib().orc_bbox_2d(_c32(Y, np.float32).ctypes.data, Y.shape[0], out.ctypes.data)
    return tuple(float(v) for v in out)


# ---------------------------------------------------------------------------------------------- FFT repulsion
def grid(Y, box_width=0.7, min_boxes=20, max_boxes=1000):
    """FFTRepulsion2D._grid (magnet/tsne.py:30-46): (xmin, ymin, width, n_boxes)."""
    xmin, ymin, xmax, ymax = bbox_2d(Y)
    lo = np.array([xmin, ymin]) - 1e-3
    hi = np.array([xmax, ymax]) + 1e-3
    span = float((hi - lo).max())
    n_boxes = int(np.clip(np.ceil(span / box_width), min_boxes, max_boxes))
    n_boxes = min(max_boxes, -(-n_boxes // 4) * 4)
    width = box_width if n_boxes * box_width >= span else max(span / n_boxes, 1e-12)
    return float(lo[0]), float(lo[1]), width, n_boxes


def kernel_spectra(n_boxes, width, n_interp=3, dof=1.0):
    """FFTRepulsion2D._kernels (magnet/tsne.py:48-71) with the .real of __call__ (:86): (M, K1h, K2h)."""
    import scipy.fft as fft
    N = n_boxes * n_interp
    M = fft.next_fast_len(2 * N, real=True)
    delta = width / n_interp
    off = np.arange(M)
    off = np.where(off <= M // 2, off, off - M).astype(np.float64) * delta
    r2 = off[:, None] ** 2 + off[None, :] ** 2
    base = 1.0 + r2 / dof
    K1 = (base ** (-dof)).astype(np.float32)
    K2 = (base ** (-dof - 1.0)).astype(np.float32)
    K1h = np.ascontiguousarray(fft.rfft2(K1), dtype=np.complex64)
    K2h = np.ascontiguousarray(fft.rfft2(K2), dtype=np.complex64)
    return int(M), np.ascontiguousarray(K1h.real), np.ascontiguousarray(K2h.real)


def fft_repulsion_fp64(Y, xmin, ymin, width, n_boxes, n_interp=3, dof=1.0):
    """The FFT-interpolated repulsion with the reference's box location and Lagrange weights, the spread and the
    gather summed in FP64 and the grid convolution done exactly (FP64 FFT, zero padded). Returns (sumQ, F)."""
    Y = _c32(Y, np.float32)
    n = Y.shape[0]
    N = n_boxes * n_interp
    W = np.empty((3, N, N), np.float64)
    lib().orc_spread(Y.ctypes.data, n, xmin, ymin, width, n_boxes, n_interp, W.ctypes.data)
    M = 2 * N
    delta = width / n_interp
    off = np.arange(M)
    off = np.where(off <= M // 2, off, off - M).astype(np.float64) * delta
    r2 = off[:, None] ** 2 + off[None, :] ** 2
    base = 1.0 + r2 / dof
    K1h = np.fft.rfft2(base ** (-dof))
    K2h = np.fft.rfft2(base ** (-dof - 1.0))
    Wh = np.fft.rfft2(W, s=(M, M), axes=(1, 2))
    phi = np.empty((4, N, N), np.float64)
    phi[0] = np.fft.irfft2(K1h * Wh[0], s=(M, M))[:N, :N]
    phi[1:] = np.fft.irfft2(K2h[None] * Wh, s=(M, M), axes=(1, 2))[:, :N, :N]
    phi = np.ascontiguousarray(phi)
    F = np.empty((n, 2), np.float64)
    sumQ = lib().orc_gather(Y.ctypes.data, n, xmin, ymin, width, n_boxes, n_interp, phi.ctypes.data, F.ctypes.data)
    return float(sumQ), F


def exact_repulsion(Y, rows=None, dof=1.0):
    """FP64 all-pairs (sumQ over the given rows, F of those rows)."""
    Y = _c32(Y, np.float32)
    n = Y.shape[0]
    r0, r1 = (0, n) if rows is None else rows
    F = np.empty((r1 - r0, 2), np.float64)
    s = lib().orc_exact_repulsion(Y.ctypes.data, n, r0, r1, float(dof), F.ctypes.data)
    return float(s), F


# ---------------------------------------------------------------------------------------------- drivers
def sampling_frequencies(w, target):
    """magnet/__init__.py:51-66."""
    w = np.asarray(w, dtype=np.float64)
    n = len(w)
    if n == 0 or n <= target:
        return np.ones_like(w)
    ws = np.sort(w)[::-1]
    tail = np.cumsum(ws[::-1])[::-1]
    t = np.arange(1, n + 1)
    s_bp = 1.0 / np.maximum(ws[t - 1], 1e-300)
    tail_t = np.append(tail[1:], 0.0)
    total = t + s_bp * tail_t
    k = int(np.searchsorted(total, target))
    s = (target - k) / tail[k] if k < n and tail[k] > 0 else s_bp[-1]
    return np.minimum(1.0, s * w)


def edge_schedule(P, n_epochs, samples_per_node=5.0):
    """magnet/__init__.py:727-737: (head, tail, epochs_per_sample) in COO order of the sorted CSR."""
    C = P.tocoo()
    w = C.data.astype(np.float64)
    freq = sampling_frequencies(w, samples_per_node * P.shape[0])
    budget = n_epochs if isinstance(n_epochs, (int, np.integer)) else 300
    keep = freq >= 1.0 / budget
    return (C.row[keep].astype(np.int32), C.col[keep].astype(np.int32), (1.0 / freq[keep]).astype(np.float32))


def optimize_sgd(Y, head, tail, eps, n_epochs, *, lr=1.0, mid_weight=0.0, mid_phase=0.5, mid_pairs=None,
                 backend="reference", n_threads=1, seed=0, a=1.577, b=0.895, rep_a=None, rep_b=1.0,
                 negative_sample_rate=5.0, repulsion_strength=2.0, mid_rate=0.25, walk_len=4, n_fixed=0,
                 indptr=None, indices=None, exaggeration=1.0):
    """MAGNET._optimize, integer-epoch path with the default late_exaggeration = 1 (one segment
    [0, n_epochs) with alpha and the mid weight interpolated linearly inside it; magnet/__init__.py:796-839).
    backend: "reference" (the compiled reference, n_threads as given) or "oracle" (the C restatement)."""
    n = Y.shape[0]
    eons = eps.copy()
    eonns = (eps / negative_sample_rate).astype(np.float32)
    total = int(n_epochs)
    mid_len = max(1.0, mid_phase * total)
    use_mid = mid_weight > 0 and ((mid_pairs is not None and mid_pairs.size > 0) or walk_len > 0) and mid_rate > 0
    alpha = lambda e: lr * (1.0 - e / total)
    mid = (lambda e: mid_weight * max(0.0, 1.0 - e / mid_len)) if use_mid else (lambda e: 0.0)
    if rep_a is None:
        rep_a = a
    mp = np.zeros((0, 1), np.int32) if mid_pairs is None else np.ascontiguousarray(mid_pairs, dtype=np.int32)
    ip = np.zeros(0, np.int32) if indptr is None else np.ascontiguousarray(indptr, np.int32)
    ix = np.zeros(0, np.int32) if indices is None else np.ascontiguousarray(indices, np.int32)
    if backend == "reference":
        R = reference()
        z32 = np.zeros(0, np.int32)
        R.optimize_layout(Y, head, tail, eps, eons, eonns, ip, ix, 0, total, float(alpha(0)), float(alpha(total)),
                          float(mid(0)), float(mid(total)), float(a), float(b), float(rep_a), float(rep_b),
                          float(negative_sample_rate), 0, float(exaggeration), float(repulsion_strength),
                          int(walk_len), float(mid_rate), 0, 0, int(n_fixed),
                          np.zeros((0, Y.shape[1]), np.float32), np.zeros((0, Y.shape[1]), np.float32), z32,
                          0.9, 0.999, z32, mp, z32, z32, 0.0, 0, np.zeros(0, np.float32), int(seed), int(n_threads), 0)
    else:
        sgd_serial(Y, head, tail, eps, eons, eonns, indptr=ip if ip.size else None, indices=ix if ix.size else None,
                   mid_pairs=mp if mp.size else None, epoch_start=0, epoch_end=total,
                   alpha0=float(alpha(0)), alpha1=float(alpha(total)), mid_w0=float(mid(0)), mid_w1=float(mid(total)),
                   a=a, b=b, rep_a=rep_a, rep_b=rep_b, negative_sample_rate=negative_sample_rate,
                   exaggeration=exaggeration, repulsion_strength=repulsion_strength, walk_len=walk_len,
                   mid_rate=mid_rate, n_fixed=n_fixed, seed=seed)
    return Y


def host_distance_order():
    """the reference's squared-distance kernel on this host (src/nndescent.cpp:101-106): 0 AVX-512, 1 AVX2 + FMA,
    2 the plain loop"""
    try:
        flags = set(open("/proc/cpuinfo").read().split())
    except OSError:
        return 2
    return 0 if "avx512f" in flags else (1 if {"avx2", "fma"} <= flags else 2)


def mid_near_pairs(X, n_pairs=5, n_cand=6, seed=0, n_threads=-1, order=None):
    """mid_near_pairs_dense (src/nndescent.cpp:731-768) restated in C: (n, n_pairs) int32. n_threads -1 means the
    host's hardware threads, as the reference resolves it; order: the distance kernel (host_distance_order())"""
    X = np.ascontiguousarray(X, dtype=np.float32)
    n, d = X.shape
    nt = n_threads if n_threads > 0 else (os.cpu_count() or 4)
    out = np.empty((n, n_pairs), np.int32)
    rc = lib().orc_mid_near_pairs(_ptr(X), n, d, int(n_pairs), int(n_cand), int(seed), int(nt),
                                  host_distance_order() if order is None else int(order), _ptr(out))
    if rc != 0:
        raise RuntimeError("need n_pairs >= 1, n_cand >= 2 and n > n_cand")
    return out


def find_ab_params(spread=1.0, min_dist=0.1):
    """magnet/__init__.py:26-48, the power kernel: a, b of 1 / (1 + a d^(2b)) fitted to the (min_dist, spread)
    curve"""
    from scipy.optimize import curve_fit
    xv = np.linspace(0, spread * 3, 300)
    yv = np.zeros(xv.shape)
    yv[xv < min_dist] = 1.0
    yv[xv >= min_dist] = np.exp(-(xv[xv >= min_dist] - min_dist) / spread)
    params, _ = curve_fit(lambda x, a, b: 1.0 / (1.0 + a * x ** (2 * b)), xv, yv)
    return float(params[0]), float(params[1])


def reference_fuzzy_graph(ind, dist, n_neighbors, n_threads=-1):
    """magnet/knn.py:215-230 on the compiled reference: its smooth_knn, then scipy's union"""
    import scipy.sparse as sp
    R = reference()
    vals = np.asarray(R.smooth_knn(np.ascontiguousarray(dist, dtype=np.float32), int(n_neighbors), 1.0, 64,
                                   int(n_threads)))
    n, k = ind.shape
    rows = np.repeat(np.arange(n, dtype=np.int64), k)
    A = sp.csr_matrix((vals.ravel(), (rows, np.asarray(ind).ravel())), shape=(n, n), dtype=np.float32)
    A.eliminate_zeros()
    T = A.T.tocsr()
    prod = A.multiply(T)
    P = (1.0 * (A + T - prod) + 0.0 * prod).tocsr()
    P.eliminate_zeros()
    P.sort_indices()
    return P


def reference_fit(X, n_neighbors=15, n_epochs=200, seed=0, n_threads=-1, a=None, b=None, mid_weight=0.1):
    """a fit on the reference's CPU path: its NN-descent kNN (magnet/knn.py:90-122), the fuzzy graph, the edge
    schedule, a PCA start rescaled to max-abs 10 (the spectral init stays out of the timed path), its mid-near
    pairs, and its SGD with the mid-range weight (MAGNET._optimize). Returns (Y, P)."""
    R = reference()
    X = np.ascontiguousarray(X, dtype=np.float32)
    n = X.shape[0]
    k = min(n_neighbors, n) - 1
    kin = min(max(k, 20), n - 1)
    n_trees = int(max(2, min(8, round(np.sqrt(n) / 40))))
    ind, d2 = R.nn_descent(X, int(kin), 50, 10, 0.001, n_trees, 30, int(seed), int(n_threads), False)
    ind = np.asarray(ind)[:, :k].astype(np.int64)
    dist = np.sqrt(np.maximum(np.asarray(d2)[:, :k], 0.0)).astype(np.float32)
    P = reference_fuzzy_graph(ind, dist, n_neighbors, n_threads)
    head, tail, eps = edge_schedule(P, n_epochs)
    rng = np.random.default_rng(seed)
    sub = X[rng.choice(n, min(n, 20000), replace=False)]
    mu = sub.mean(0)
    _, _, Vt = np.linalg.svd(sub - mu, full_matrices=False)
    Y = ((X - mu) @ Vt[:2].T).astype(np.float32)
    Y = np.ascontiguousarray(10.0 * Y / np.abs(Y).max(), dtype=np.float32)
    pairs = np.asarray(R.mid_near_pairs_dense(X, 5, 6, int(seed), int(n_threads)))
    if a is None or b is None:
        a, b = find_ab_params(1.0, 0.1)
    optimize_sgd(Y, head, tail, eps, n_epochs, mid_weight=mid_weight, mid_pairs=pairs, backend="reference",
                 n_threads=n_threads, seed=seed, a=a, b=b, indptr=P.indptr, indices=P.indices)
    return Y, P


def choose_landmarks(n, random_state=0):
    """magnet/knn.py:125-128"""
    m = int(min(n, max(100, 4 * np.sqrt(n))))
    return np.sort(np.random.default_rng(random_state).choice(n, m, replace=False)).astype(np.int32)


def transform_step(Y_train):
    """the transform step scale of magnet/__init__.py:899-906: min(1, median 1-NN spacing / 0.14)"""
    from sklearn.neighbors import NearestNeighbors
    n = Y_train.shape[0]
    sub = Y_train[np.random.default_rng(0).choice(n, min(n, 5000), replace=False)]
    d1 = float(np.median(NearestNeighbors(n_neighbors=2).fit(Y_train).kneighbors(sub)[0][:, 1]))
    return float(min(1.0, d1 / 0.14))


def reference_transform(X_train, P, Y_train, landmarks, step, Q, *, a, b, n_neighbors=15, n_epochs=100, seed=0,
                        n_threads=-1):
    """MAGNET.transform (magnet/__init__.py:876-930) on the reference's CPU path: its beam search over the
    training graph (knn_search, magnet/knn.py:131-152), smooth_knn, the start at the membership-weighted mean,
    the schedule, and its SGD with the training rows fixed at the spacing-scaled step"""
    R = reference()
    n_train = Y_train.shape[0]
    k = min(n_neighbors, n_train) - 1
    Q = np.ascontiguousarray(Q, dtype=np.float32)
    ind, d2 = R.knn_search(X_train, P.indptr.astype(np.int32), P.indices.astype(np.int32), landmarks, Q, int(k),
                           int(max(64, 2 * k + 10)), 5, int(seed), int(n_threads))
    ind = np.asarray(ind).astype(np.int64)
    dist = np.sqrt(np.maximum(np.asarray(d2), 0.0)).astype(np.float32)
    vals = np.asarray(R.smooth_knn(dist, int(n_neighbors), 1.0, 64, int(n_threads)))
    W = vals / np.maximum(vals.sum(1, keepdims=True), 1e-12)
    Y_new = np.einsum("mk,mkd->md", W, Y_train[ind]).astype(np.float32)
    m = Q.shape[0]
    Y_all = np.ascontiguousarray(np.vstack([Y_train, Y_new]), dtype=np.float32)
    freq = sampling_frequencies(vals.ravel().astype(np.float64), 5.0 * m)
    keep = freq >= 1.0 / n_epochs
    head = (n_train + np.repeat(np.arange(m), k)).astype(np.int32)[keep]
    tail = ind.ravel().astype(np.int32)[keep]
    eps = (1.0 / freq[keep]).astype(np.float32)
    optimize_sgd(Y_all, head, tail, eps, n_epochs, lr=step, backend="reference", n_threads=n_threads, seed=seed,
                 a=a, b=b, n_fixed=n_train)
    return Y_all[n_train:]


class TsneRun:
    """The loop of magnet/tsne.py:132-184 (the common path: no mid-range or far-field terms) as a resumable run:
    the set-up of the reference's driver (P normalised to sum 1, the learning rate, zero update, unit gains, the
    spectrum and FFTConv2D caches) once, then ``advance(k)`` runs the next k iterations with the same state, so a
    long pass can be timed in pieces. backend "reference" drives the compiled reference's kernels, "oracle" the C
    restatement with the FP64 convolution."""

    def __init__(self, P, Y, n_iter=750, early_iter=250, early_exaggeration=12.0, exaggeration=1.0,
                 learning_rate=None, momentum=(0.5, 0.8), n_interp=3, box_width=0.7, n_threads=-1, dof=1.0,
                 backend="reference", callback=None):
        import scipy.sparse as sp
        n = P.shape[0]
        P = sp.csr_matrix(P, dtype=np.float32)
        P = P / P.sum()
        self.indptr, self.indices, self.data = (P.indptr.astype(np.int32), P.indices.astype(np.int32),
                                                P.data.astype(np.float32))
        self.lr = max(200.0, n / early_exaggeration) if learning_rate is None else learning_rate
        self.Y = np.ascontiguousarray(Y, dtype=np.float32)
        self.update = np.zeros_like(self.Y)
        self.gains = np.ones_like(self.Y)
        self.R = reference() if backend == "reference" else None
        self.convs, self.spectra = {}, {}
        self.it = 0
        self.n_iter, self.early_iter = n_iter, early_iter
        self.early_exaggeration, self.exaggeration, self.momentum = early_exaggeration, exaggeration, momentum
        self.n_interp, self.box_width, self.n_threads, self.dof = n_interp, box_width, n_threads, dof
        self.callback = callback

    def advance(self, k):
        """runs iterations it .. min(it + k, n_iter) - 1; returns Y (updated in place)"""
        R, Y, update, gains = self.R, self.Y, self.update, self.gains
        indptr, indices, data = self.indptr, self.indices, self.data
        n_interp, box_width, n_threads, dof = self.n_interp, self.box_width, self.n_threads, self.dof
        for it in range(self.it, min(self.it + k, self.n_iter)):
            early = it < self.early_iter
            rho = self.early_exaggeration if early else self.exaggeration
            mom = self.momentum[0] if early else self.momentum[1]
            if R is not None:
                attr = np.asarray(R.tsne_attraction(indptr, indices, data, Y, float(dof), n_threads))
                xmin, ymin, xmax, ymax = R.bbox_2d(Y, n_threads)
                lo = np.array([xmin, ymin]) - 1e-3
                hi = np.array([xmax, ymax]) + 1e-3
                span = float((hi - lo).max())
                n_boxes = int(np.clip(np.ceil(span / box_width), 20, 1000))
                n_boxes = min(1000, -(-n_boxes // 4) * 4)
                width = box_width if n_boxes * box_width >= span else max(span / n_boxes, 1e-12)
                key = (n_boxes, round(width, 6))
                if key not in self.spectra:
                    if len(self.spectra) > 8:
                        self.spectra.pop(next(iter(self.spectra)))
                    self.spectra[key] = kernel_spectra(n_boxes, width, n_interp, dof)
                M, K1, K2 = self.spectra[key]
                ck = (M, round(width, 6))
                conv = self.convs.get(ck)
                if conv is None:
                    conv = R.FFTConv2D(int(M), n_interp)
                    conv.set_kernels(K1, K2)
                    if len(self.convs) > 4:
                        self.convs.pop(next(iter(self.convs)))
                    self.convs[ck] = conv
                sumQ, F = conv.compute(Y, float(lo[0]), float(lo[1]), width, n_boxes, n_threads)
                R.tsne_step(Y, update, gains, attr, np.asarray(F), float(rho), float(1.0 / max(sumQ, 1e-12)),
                            float(self.lr), float(mom), n_threads)
            else:
                attr = tsne_attraction(indptr, indices, data, Y, dof)
                xmin, ymin, width, n_boxes = grid(Y, box_width)
                sumQ, F = fft_repulsion_fp64(Y, xmin, ymin, width, n_boxes, n_interp, dof)
                tsne_step(Y, update, gains, attr, F.astype(np.float32), float(rho), float(1.0 / max(sumQ, 1e-12)),
                          float(self.lr), float(mom))
            if self.callback is not None:
                self.callback(it, Y)
        self.it = min(self.it + k, self.n_iter)
        return Y


def optimize_tsne(P, Y, n_iter=750, early_iter=250, early_exaggeration=12.0, exaggeration=1.0,
                  learning_rate=None, momentum=(0.5, 0.8), n_interp=3, box_width=0.7, n_threads=-1,
                  dof=1.0, backend="reference", callback=None):
    """magnet/tsne.py:132-184 (the common path: no mid-range or far-field terms), driving the compiled
    reference's kernels (backend "reference") or the C restatement with the FP64 convolution ("oracle")."""
    run = TsneRun(P, Y, n_iter, early_iter, early_exaggeration, exaggeration, learning_rate, momentum, n_interp,
                  box_width, n_threads, dof, backend, callback)
    return run.advance(n_iter)


# ---------------------------------------------------------------------------------------------- spectral init
def _jacobi_eigen(H):
    """cyclic Jacobi rotations on a small symmetric matrix (Golub and Van Loan, section 8.5), as
    src/spectral.cpp:87-123 runs them: eigenvalues descending, eigenvectors as columns"""
    A = np.array(H, dtype=np.float64)
    p = A.shape[0]
    V = np.eye(p)
    for _ in range(100):
        if sum(A[i, j] ** 2 for i in range(p) for j in range(i + 1, p)) < 1e-22:
            break
        for i in range(p):
            for j in range(i + 1, p):
                aij = A[i, j]
                if abs(aij) < 1e-300:
                    continue
                th = (A[j, j] - A[i, i]) / (2.0 * aij)
                t = (1.0 if th >= 0 else -1.0) / (abs(th) + np.sqrt(th * th + 1.0))
                c = 1.0 / np.sqrt(t * t + 1.0)
                s = t * c
                for M in (A, V):
                    x, y = M[:, i].copy(), M[:, j].copy()
                    M[:, i], M[:, j] = c * x - s * y, s * x + c * y
                x, y = A[i, :].copy(), A[j, :].copy()
                A[i, :], A[j, :] = c * x - s * y, s * x + c * y
    d = np.diag(A).copy()
    order = sorted(range(p), key=lambda k: -d[k])
    return d[order], V[:, order]


def chebyshev_eigenvectors(indptr, indices, data, X, inv_sqrt_deg, component, n_wanted, degree, max_iter, tol):
    """src/spectral.cpp:141-241 in numpy (FP64): the Chebyshev-filtered subspace iteration with Rayleigh-Ritz for
    the leading non-trivial eigenvectors of (I + D^-1/2 A D^-1/2) / 2, the trivial eigenvector deflated per
    connected component, two passes of modified Gram-Schmidt; returns the float32 block"""
    import scipy.sparse as sp
    n, p = X.shape
    A = sp.csr_matrix((np.asarray(data, np.float64), indices, indptr), shape=(n, n))
    sd = np.asarray(inv_sqrt_deg, np.float64)
    comp = np.asarray(component, np.int64)
    t = np.where(sd > 0, 1.0 / np.where(sd > 0, sd, 1.0), 0.0)
    nc = int(comp.max()) + 1
    tn = np.bincount(comp, weights=t * t, minlength=nc)

    def M(Y):
        return 0.5 * (Y + sd[:, None] * (A @ (sd[:, None] * Y)))

    def deflate(Y):
        pr = np.stack([np.bincount(comp, weights=t * Y[:, k], minlength=nc) for k in range(p)], 1)
        pr = np.where(tn[:, None] > 0, pr / np.where(tn[:, None] > 0, tn[:, None], 1.0), 0.0)
        return Y - t[:, None] * pr[comp]

    def orthonormalize(Y):
        for _ in range(2):
            for k in range(p):
                for j in range(k):
                    Y[:, k] -= (Y[:, k] @ Y[:, j]) * Y[:, j]
                nrm = Y[:, k] @ Y[:, k]
                Y[:, k] *= 1.0 / np.sqrt(nrm) if nrm > 1e-300 else 0.0
        return Y

    def rayleigh_ritz(X):
        Z = deflate(M(X))
        H = X.T @ Z
        H = np.triu(H) + np.triu(H, 1).T
        theta, V = _jacobi_eigen(H)
        X, Z = X @ V, Z @ V
        return X, Z, theta, max(np.linalg.norm(Z[:, c] - theta[c] * X[:, c]) for c in range(n_wanted))

    X = orthonormalize(deflate(np.asarray(X, np.float64)))
    X, Z, theta, res = rayleigh_ritz(X)
    prev = -1.0
    for _ in range(max_iter):
        gap = max(theta[n_wanted - 1] - theta[n_wanted], 1e-3)
        total = theta[:n_wanted].sum()
        if res < tol * gap or res < 1e-9 or (prev >= 0 and abs(total - prev) < 1e-9 * n_wanted):
            break
        prev = total
        alpha = max(min(theta[p - 1], theta[n_wanted - 1] - 0.5 * gap), 1e-3)
        a0 = min(1.0, theta[0] + 1e-9)
        e = cc = 0.5 * alpha
        s1 = e / (a0 - cc)
        sigma = s1
        Y = (deflate(M(X)) - cc * X) * (s1 / e)
        for _ in range(2, degree + 1):
            sn = 1.0 / (2.0 / s1 - sigma)
            Yn = (deflate(M(Y)) - cc * Y) * (2.0 * sn / e) - sigma * sn * X
            X, Y, sigma = Y, Yn, sn
        X = orthonormalize(deflate(Y.copy()))
        X, Z, theta, res = rayleigh_ritz(X)
    return X.astype(np.float32)
