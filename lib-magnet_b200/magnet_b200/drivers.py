"""Python drivers of the layout pass, mirroring the reference's drivers over the device entry points.

Each function keeps the reference's signature and semantics (cited per function); the arithmetic runs on the
device through ``magnet_b200._native``. Arrays may be numpy (copied to and from the device by the call, updated
in place like the reference) or device tensors exposing ``__cuda_array_interface__`` (used in place).
"""
import numpy as np
import scipy.sparse as sp

from . import _native as N


def find_ab_params(spread=1.0, min_dist=0.1, b=None, kernel="power"):
    """Fit of the low-dimensional kernel to the (min_dist, spread) curve (magnet/__init__.py:26-48): 1/(1 + a d^2b)
    ("power"; a and b, or only a when b is given), exp(-a d^2) ("gaussian"), 1/cosh(a d) ("sech"),
    1 - tanh(a d^2) ("tanh")."""
    from scipy.optimize import curve_fit

    xv = np.linspace(0, spread * 3, 300)
    yv = np.zeros(xv.shape)
    yv[xv < min_dist] = 1.0
    yv[xv >= min_dist] = np.exp(-(xv[xv >= min_dist] - min_dist) / spread)
    curves = {"gaussian": lambda x, a: np.exp(-a * x ** 2), "sech": lambda x, a: 1.0 / np.cosh(a * x),
              "tanh": lambda x, a: 1.0 - np.tanh(a * x ** 2)}
    if kernel in curves:
        params, _ = curve_fit(curves[kernel], xv, yv, p0=[1.0])
        return float(params[0]), 1.0
    if b is None:
        params, _ = curve_fit(lambda x, a, bb: 1.0 / (1.0 + a * x ** (2 * bb)), xv, yv)
        return float(params[0]), float(params[1])
    params, _ = curve_fit(lambda x, a: 1.0 / (1.0 + a * x ** (2 * b)), xv, yv, p0=[1.0])
    return float(params[0]), float(b)


# ---------------------------------------------------------------------------------------------- FFT repulsion
class FFTRepulsion2D:
    """Potentials sum_j K(|y_i - y_j|) c_j of the two t-SNE kernels by Lagrange interpolation on boxes of fixed
    width and an FFT convolution of the equispaced nodes, on the device (magnet/tsne.py:11-90): the same grid
    choice (_grid), the same kernel spectra cached per grid (_kernels) and one persistent device FFTConv2D per
    (M, width). Returns (sumQ, F) with F a numpy array for numpy input and a device tensor for device input."""

    def __init__(self, n_interp=3, box_width=0.7, min_boxes=20, max_boxes=1000, n_threads=-1, dof=1.0, kernels=None):
        self.dof = float(dof)
        self.kernels = kernels
        self.n_interp = n_interp
        self.box_width = box_width
        self.min_boxes = min_boxes
        self.max_boxes = max_boxes
        self.n_threads = n_threads
        self._cache = {}
        self._convs = {}

    def _grid(self, Y):
        xmin, ymin, xmax, ymax = N.bbox_2d(Y, self.n_threads)
        lo = np.array([xmin, ymin]) - 1e-3
        hi = np.array([xmax, ymax]) + 1e-3
        span = float((hi - lo).max())
        n_boxes = int(np.clip(np.ceil(span / self.box_width), self.min_boxes, self.max_boxes))
        n_boxes = min(self.max_boxes, -(-n_boxes // 4) * 4)
        width = self.box_width if n_boxes * self.box_width >= span else max(span / n_boxes, 1e-12)
        return float(lo[0]), float(lo[1]), width, n_boxes

    def _kernels(self, n_boxes, width):
        import scipy.fft as fft
        key = (n_boxes, round(width, 6))
        if key not in self._cache:
            if len(self._cache) > 8:
                self._cache.pop(next(iter(self._cache)))
            Nn = n_boxes * self.n_interp
            M = fft.next_fast_len(2 * Nn, real=True)
            delta = width / self.n_interp
            off = np.arange(M)
            off = np.where(off <= M // 2, off, off - M).astype(np.float64) * delta
            r2 = off[:, None] ** 2 + off[None, :] ** 2
            if self.kernels is not None:
                K1, K2 = self.kernels(r2)
                K1 = np.asarray(K1, dtype=np.float32); K2 = np.asarray(K2, dtype=np.float32)
            else:
                base = 1.0 + r2 / self.dof
                K1 = (base ** (-self.dof)).astype(np.float32)
                K2 = (base ** (-self.dof - 1.0)).astype(np.float32)
            self._cache[key] = (M, np.ascontiguousarray(fft.rfft2(K1), dtype=np.complex64),
                                np.ascontiguousarray(fft.rfft2(K2), dtype=np.complex64))
        return self._cache[key]

    def __call__(self, Y):
        if not hasattr(Y, "__cuda_array_interface__"):
            Y = np.ascontiguousarray(Y, dtype=np.float32)
        xmin, ymin, width, n_boxes = self._grid(Y)
        M, K1h, K2h = self._kernels(n_boxes, width)
        conv = self._convs.get((int(M), round(width, 6)))
        if conv is None:
            conv = N.FFTConv2D(int(M), self.n_interp)
            conv.set_kernels(np.ascontiguousarray(K1h.real), np.ascontiguousarray(K2h.real))
            if len(self._convs) > 4:
                self._convs.pop(next(iter(self._convs)))
            self._convs[(int(M), round(width, 6))] = conv
        sumQ, F = conv.compute(Y, xmin, ymin, width, n_boxes, self.n_threads)
        return float(sumQ), F


def _csr32(P):
    P = sp.csr_matrix(P, dtype=np.float32)
    return P.indptr.astype(np.int32), P.indices.astype(np.int32), P.data.astype(np.float32)


def optimize_tsne(P, Y, n_iter=750, early_iter=250, early_exaggeration=12.0, exaggeration=1.0,
                  learning_rate=None, momentum=(0.5, 0.8), n_interp=3, box_width=0.7, n_threads=-1,
                  mid_pairs=None, mid_weight=0.0, mid_phase=0.5, dof=1.0, verbose=False, callback=None,
                  far_weight=0.0, far_r0=0.1, far_a=1.74, mid_form="mean", mid_c=0.3, threads_per_row=0,
                  use_graph=True):
    """Full-batch t-SNE gradient descent (magnet/tsne.py:132-214). P: symmetric CSR affinities (normalised to
    sum 1 inside), Y: (n, 2) float32 initial layout, updated in place and returned.

    The common path (no mid-range or far-field term, no callback) runs entirely on the device, each iteration a
    replay of one captured CUDA graph. With mid-range pairs, a far-field term or a callback, the reference's
    per-iteration sequence runs instead (attraction, FFT repulsion, mid spring, update), each step on the
    device."""
    n = P.shape[0]
    if learning_rate is None:
        learning_rate = max(200.0, n / early_exaggeration)
    on_device = hasattr(Y, "__cuda_array_interface__")
    if not on_device:
        Y = np.ascontiguousarray(Y, dtype=np.float32)
    common = far_weight <= 0 and (mid_pairs is None or mid_weight <= 0) and callback is None
    if common:
        ip, ix, dd = _csr32(P)
        N.optimize_tsne(ip, ix, dd, Y, int(n_iter), int(early_iter), float(early_exaggeration), float(exaggeration),
                        float(learning_rate), float(momentum[0]), float(momentum[1]), int(n_interp),
                        float(box_width), float(dof), 20, 1000, int(threads_per_row), bool(use_graph))
        return Y
    Pn = sp.csr_matrix(P, dtype=np.float32)
    Pn = Pn / Pn.sum()
    ip, ix, dd = _csr32(Pn)
    if on_device:
        raise ValueError("the mid-range / far-field / callback path takes numpy layouts")
    if mid_pairs is not None:
        mid_pairs = np.ascontiguousarray(mid_pairs, dtype=np.int32)
    update = np.zeros_like(Y)
    gains = np.ones_like(Y)
    rep = FFTRepulsion2D(n_interp=n_interp, box_width=box_width, n_threads=n_threads, dof=dof)
    rep_far, r0_cur = None, None

    def make_far(r0):
        r02 = float(r0) ** 2
        return FFTRepulsion2D(n_interp=n_interp, box_width=box_width, n_threads=n_threads,
                              kernels=lambda r2: (np.zeros_like(r2), 2.0 * r2 ** 4 / ((1.0 + far_a * r2) ** 5 * (r02 + r2))))

    for it in range(n_iter):
        early = it < early_iter
        rho = early_exaggeration if early else exaggeration
        mom = momentum[0] if early else momentum[1]
        attr = np.asarray(N.tsne_attraction(ip, ix, dd, Y, float(dof), n_threads))
        sumQ, F = rep(Y)
        grad = rho * attr
        grad -= F * (1.0 / max(sumQ, 1e-12))
        if far_weight > 0 and not early:
            if it % 25 == 0 or rep_far is None:
                r0_new = far_r0 * float(np.sqrt(((Y - Y.mean(0)) ** 2).sum(1).mean()))
                if r0_cur is None or abs(r0_new - r0_cur) > 0.2 * r0_cur:
                    rep_far, r0_cur = make_far(r0_new), r0_new
            _, F_far = rep_far(Y)
            grad -= far_weight * F_far
        if mid_pairs is not None and mid_weight > 0:
            w_mid = mid_weight * max(0.0, 1.0 - it / max(1.0, mid_phase * n_iter)) / n
            if w_mid > 0 and mid_form == "mean":
                grad = np.ascontiguousarray(grad, dtype=np.float32)
                N.mid_spring(Y, mid_pairs, grad, float(w_mid), n_threads)
            elif w_mid > 0:
                c2 = (mid_c * float(np.sqrt(((Y - Y.mean(0)) ** 2).sum(1).mean()))) ** 2
                for k in range(mid_pairs.shape[1]):
                    diff = Y - Y[mid_pairs[:, k]]
                    grad += (w_mid / mid_pairs.shape[1]) * diff / (1.0 + (diff ** 2).sum(1, keepdims=True) / c2)
        N.tsne_update(Y, update, gains, np.ascontiguousarray(grad, dtype=np.float32), float(learning_rate),
                      float(mom), n_threads)
        if callback is not None and (it % 50 == 0 or it == n_iter - 1):
            callback(it, Y)
    return Y


def optimize_tsne_batch(Ps, Ys, n_iter=500, early_iter=None, early_exaggeration=12.0, exaggeration=1.0,
                        learning_rate=None, momentum=(0.5, 0.8), n_interp=3, box_width=0.7, dof=1.0,
                        max_boxes=None, threads_per_row=None, branches=None, autotune=True):
    """Many independent t-SNE passes (each the device loop of optimize_tsne, magnet/tsne.py:132-214) run together:
    one CUDA graph holds one iteration of every layout as independent branches, replayed n_iter times. Ps: the
    layouts' symmetric CSR affinities (each normalised to sum 1 inside), Ys: their (n_i, 2) float32 initial layouts
    (numpy or device arrays), updated in place and returned. early_iter None: min(250, n_iter // 3), MAGNET's
    default for loss="tsne" (magnet/__init__.py:640). The learning rate, when None, is each layout's own
    max(200, n_i / 12).

    threads_per_row / branches None: the autotuner's cached choice for this batch's shape (magnet_b200.autotune),
    tuned now when autotune is True and nothing is cached, else 8 lanes chosen from the row length and 32 branches.
    max_boxes: per-layout grid allocation (None: 64 + 2 ceil(sqrt(n_i)))."""
    from . import autotune as A
    if early_iter is None:
        early_iter = min(250, int(n_iter) // 3)
    graphs = [_csr32(P) for P in Ps]
    Ys = [Y if hasattr(Y, "__cuda_array_interface__") else np.ascontiguousarray(Y, dtype=np.float32) for Y in Ys]
    params = dict(early_iter=int(early_iter), early_exaggeration=float(early_exaggeration),
                  exaggeration=float(exaggeration), momentum_early=float(momentum[0]),
                  momentum_late=float(momentum[1]), n_interp=int(n_interp), box_width=float(box_width),
                  dof=float(dof), layout_max_boxes=None if max_boxes is None else [int(b) for b in max_boxes])
    if learning_rate is not None:
        params["learning_rate"] = float(learning_rate)
    if threads_per_row is None or branches is None:
        key = A.batch_key([g[0].size - 1 for g in graphs], [g[1].size for g in graphs])
        choice = A.lookup(key)
        if choice is None and autotune:
            choice = A.tune_tsne_batch(graphs, Ys, params, key=key)
        choice = choice or {"threads_per_row": 0, "branches": 32}
        threads_per_row = choice["threads_per_row"] if threads_per_row is None else threads_per_row
        branches = choice["branches"] if branches is None else branches
    batch = N.TsneBatch(graphs, n_iter=int(n_iter), threads_per_row=int(threads_per_row), branches=int(branches),
                        **params)
    batch.run(Ys)
    return Ys


# ---------------------------------------------------------------------------------------------- SGD
def sampling_frequencies(w, target):
    """freq_i = min(1, s w_i) with s solved exactly so that sum(freq) == target (magnet/__init__.py:51-66)."""
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


def edge_schedule(P, n_epochs, samples_per_node=5.0, device=False):
    """Edges sampled every 1 / min(1, s w_i) epochs, s giving samples_per_node * n samples per epoch; edges visited
    less than once dropped (magnet/__init__.py:727-737). Returns (head, tail, epochs_per_sample) in the COO order
    of the CSR (sorted by head). device=True solves s on the device (mg_edge_schedule): the same edges, eps equal
    up to FP64 rounding of s; the host path is the reference's arithmetic bit for bit."""
    budget = n_epochs if isinstance(n_epochs, (int, np.integer)) else 300
    if device:
        from . import _native as N
        P = sp.csr_matrix(P)
        return N.edge_schedule_device(P.indptr.astype(np.int32), P.indices.astype(np.int32),
                                      P.data.astype(np.float32), int(budget), float(samples_per_node))
    C = sp.csr_matrix(P).tocoo()
    w = C.data.astype(np.float64)
    freq = sampling_frequencies(w, samples_per_node * P.shape[0])
    keep = freq >= 1.0 / budget
    return C.row[keep].astype(np.int32), C.col[keep].astype(np.int32), (1.0 / freq[keep]).astype(np.float32)


def optimize_sgd(Y, head, tail, epochs_per_sample, n_epochs, *, a, b, rep_a=None, rep_b=1.0, learning_rate=1.0,
                 mid_weight=0.0, mid_phase=0.5, mid_pairs=None, graph=None, walk_len=4, mid_rate=0.25,
                 negative_sample_rate=5.0, repulsion_strength=2.0, exaggeration=1.0, late_exaggeration=1.0,
                 late_phase=0.2, loss=0, kernel=0, optimizer=0, clip=0, n_fixed=0, seed=0, stream_mode=0,
                 node_b=None, beta1=0.9, beta2=0.999, parallel="hogwild", jump_graph=None, mid_jump=0.5,
                 walk_lens=None):
    """The sampled SGD pass of MAGNET._optimize (magnet/__init__.py:751-839, integer n_epochs): eons / eonns
    initialised from the schedule, linear learning-rate decay lr (1 - e / total), mid-range weight
    mid_weight max(0, 1 - e / (mid_phase total)), segments at the late-exaggeration boundary, each segment one
    device optimize_layout call. Y is updated in place.

    parallel: "hogwild" (the device's draws per stream_mode), "serial" (the reference's single stream replayed
    exactly, stream_mode 1) or "owner" (the reference's owner mode, magnet/__init__.py:758-761, 789-794: with
    mid-near pairs and no jump graph, each node also receives the pulls of the nodes that chose it).
    jump_graph: CSR of mid-range jumps taken with probability mid_jump on each walk step; walk_lens: per-node walk
    lengths (magnet/__init__.py:774-786)."""
    if parallel not in ("hogwild", "owner", "serial"):
        raise ValueError("parallel must be 'hogwild', 'serial' or 'owner'")
    if parallel == "owner" and loss == 1:
        raise ValueError("parallel='owner' is not available with loss='infonce' (the negatives are moved)")
    n, dim = Y.shape
    total = int(n_epochs)
    lr = float(learning_rate)
    mid_pairs = np.zeros((0, 1), np.int32) if mid_pairs is None else np.ascontiguousarray(mid_pairs, dtype=np.int32)
    use_mid = mid_weight > 0 and (walk_len > 0 or mid_pairs.size > 0) and mid_rate > 0 and \
        (graph is not None or mid_pairs.size > 0)
    if use_mid and graph is not None:
        G = sp.csr_matrix(graph)
        indptr, indices = G.indptr.astype(np.int32), G.indices.astype(np.int32)
    else:
        indptr = indices = np.zeros(0, np.int32)
    eons = np.ascontiguousarray(epochs_per_sample, dtype=np.float32).copy()
    eonns = (np.asarray(epochs_per_sample, dtype=np.float32) / negative_sample_rate).astype(np.float32)
    if rep_a is None:
        rep_a = a
    z32 = np.zeros(0, np.int32)
    if optimizer == 1:
        am = np.zeros((n, dim), np.float32); av = np.zeros((n, dim), np.float32); at = np.zeros(n, np.int32)
    else:
        am = av = np.zeros((0, dim), np.float32); at = z32
    nb = np.zeros(0, np.float32) if node_b is None else np.ascontiguousarray(node_b, dtype=np.float32)
    if jump_graph is not None:
        J = sp.csr_matrix(jump_graph)
        jp, jx, mj = J.indptr.astype(np.int32), J.indices.astype(np.int32), float(mid_jump)
    else:
        jp, jx, mj = z32, z32, 0.0
    wl = z32 if walk_lens is None or not use_mid else np.ascontiguousarray(walk_lens, dtype=np.int32)
    rp = rx = z32
    if parallel == "owner" and mid_pairs.size > 0 and jump_graph is None:
        m = mid_pairs.shape[1]
        R = sp.csr_matrix((np.ones(mid_pairs.size, np.float32), (mid_pairs.ravel(), np.repeat(np.arange(n), m))),
                          shape=(n, n))
        R.sort_indices()
        rp, rx = R.indptr.astype(np.int32), R.indices.astype(np.int32)
    par = 1 if parallel == "owner" else 0
    if parallel == "serial":
        stream_mode = 1
    mid_len = max(1.0, mid_phase * total)
    alpha = lambda e: lr * (1.0 - e / total)
    mid = (lambda e: mid_weight * max(0.0, 1.0 - e / mid_len)) if use_mid else (lambda e: 0.0)
    late_start = total - int(round(late_phase * total)) if late_exaggeration != 1.0 else total
    bounds = sorted(set([0, total, late_start]))
    for e0, e1 in zip(bounds[:-1], bounds[1:]):
        if e1 <= e0:
            continue
        exag = exaggeration * late_exaggeration if e0 >= late_start else exaggeration
        N.optimize_layout(Y, head, tail, epochs_per_sample, eons, eonns, indptr, indices, int(e0), int(e1),
                          float(alpha(e0)), float(alpha(e1)), float(mid(e0)), float(mid(e1)), float(a), float(b),
                          float(rep_a), float(rep_b), float(negative_sample_rate), int(loss), float(exag),
                          float(repulsion_strength), int(walk_len), float(mid_rate), int(optimizer), int(clip),
                          int(n_fixed), am, av, at, float(beta1), float(beta2), wl, mid_pairs, jp, jx, mj,
                          int(kernel), nb, int(seed), -1, par, rp, rx, int(stream_mode))
    return Y


def hybrid_layout(P, Y, *, a, b, rep_a=None, rep_b=1.0, n_epochs=None, mid_pairs=None, mid_weight=0.2, seed=0,
                  hybrid_iter=300, n_interp=3, box_width=0.7, dof=1.0, exaggeration=1.0, stream_mode=0,
                  learning_rate=1.0):
    """loss="hybrid" (magnet/__init__.py:662-708): the sampled SGD pass (mid weight 0.2 by default), then the
    layout recentred and rescaled to std 31 sqrt(n / 70000) and refined by hybrid_iter iterations of the
    full-batch pass without early exaggeration. Y (n, 2) float32, updated and returned."""
    n = P.shape[0]
    if n_epochs is None:
        n_epochs = 500 if n <= 10000 else (300 if n <= 100000 else 200)
    head, tail, eps = edge_schedule(P, n_epochs)
    optimize_sgd(Y, head, tail, eps, n_epochs, a=a, b=b, rep_a=rep_a, rep_b=rep_b, mid_weight=mid_weight,
                 mid_pairs=mid_pairs, graph=P, seed=seed, stream_mode=stream_mode, learning_rate=learning_rate)
    Y -= Y.mean(0)
    Y *= 31.0 * np.sqrt(n / 70000.0) / max(float(Y[:, 0].std()), 1e-12)
    optimize_tsne(P, Y, n_iter=int(hybrid_iter), early_iter=0, exaggeration=exaggeration, n_interp=n_interp,
                  box_width=box_width, dof=dof)
    return Y


def transform_layout(Y_train, ind, vals, *, a, b, rep_a=None, rep_b=1.0, n_epochs=200, learning_rate=1.0,
                     step_scale=None, samples_per_node=5.0, seed=0, stream_mode=0):
    """Out-of-sample placement of MAGNET.transform (magnet/__init__.py:896-930) from the new points' neighbours
    in the training set: ind (m, k) training indices, vals (m, k) smooth-kNN memberships. New points start at
    the membership-weighted mean of their neighbours and are optimised for n_epochs with the training points
    fixed (n_fixed), at the learning rate learning_rate * step_scale (the layout-spacing step of the reference,
    min(1, d1 / 0.14); computed from Y_train when None). Returns the (m, dim) new positions."""
    Y_train = np.ascontiguousarray(Y_train, dtype=np.float32)
    n_train, dim = Y_train.shape
    m, k = ind.shape
    W = vals / np.maximum(vals.sum(1, keepdims=True), 1e-12)
    Y_new = np.einsum("mk,mkd->md", W, Y_train[ind]).astype(np.float32)
    Y_all = np.ascontiguousarray(np.vstack([Y_train, Y_new]), dtype=np.float32)
    if step_scale is None:
        rng = np.random.default_rng(0)
        sub = Y_train[rng.choice(n_train, min(n_train, 5000), replace=False)]
        from scipy.spatial import cKDTree
        d1 = float(np.median(cKDTree(Y_train).query(sub, k=2)[0][:, 1]))
        step_scale = float(min(1.0, d1 / 0.14))
    w = np.asarray(vals, dtype=np.float64).ravel()
    freq = sampling_frequencies(w, samples_per_node * m)
    keep = freq >= 1.0 / n_epochs
    head = (n_train + np.repeat(np.arange(m), k)).astype(np.int32)[keep]
    tail = np.asarray(ind).ravel().astype(np.int32)[keep]
    eps = (1.0 / freq[keep]).astype(np.float32)
    optimize_sgd(Y_all, head, tail, eps, int(n_epochs), a=a, b=b, rep_a=rep_a, rep_b=rep_b,
                 learning_rate=learning_rate * step_scale, mid_weight=0.0, n_fixed=n_train, seed=seed,
                 stream_mode=stream_mode)
    return Y_all[n_train:]
