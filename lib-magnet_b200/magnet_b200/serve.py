"""Continuous-batching layout server on one device: a fitted layout stays resident in HBM, transform() requests
(MAGNET.transform, magnet/__init__.py:876-930) and fit requests (MAGNET.fit) are admitted as they arrive, as
slots and device memory free up, and their work overlaps on the device.

* ``Server``: the scheduler. Requests wait in one FIFO; ``slots`` worker threads take them in order, each after
  reserving the request's device bytes from a budget (admission by free memory), in the order they were taken;
  a request that does not fit waits until running ones release theirs, and later requests wait behind it. The
  work itself is a function of the request, so the scheduler is independent of the device (it is tested on the
  host with plain functions).
* ``FittedLayout``: the resident training data X (n, d), its layout Y (n, 2) and the kernel constants.
  ``transform`` places new rows as the reference does: their k = n_neighbors - 1 nearest training rows by the
  reference's beam search over the training rows' neighbour graph from the closest landmarks (on the device,
  mg_knn_search; exact blocked matmul when no graph is given), smooth_knn memberships (device), the start at the
  membership-weighted mean of the neighbours' positions,
  the reference's edge schedule and step scale, then the SGD with the training rows fixed (n_fixed), on the
  device. Owner mode (parallel='owner', the default here) makes a request's result a function of its inputs
  alone, so it is the same bits alone and in any mix; parallel='hogwild' agrees to float rounding. The owner
  chunks are 256 edges (owner_chunk_edges) instead of the reference's 4096: a transform has few edges, and
  each chunk is one serial stream, so smaller chunks run more streams side by side. The result is
  deterministic but does not reproduce the reference's owner-mode streams. The reference's own transform runs
  hogwild, which has no reproducible streams either.
* ``fit_layout``: a fit request (exact kNN, fuzzy graph, edge schedule, PCA start, SGD), on the device.

Each worker thread owns a CUDA stream: torch work runs on it and the C ABI is pointed at it (mg_set_stream is
per thread), so requests in different slots overlap and never share device scratch (the library's staging and
SGD buffers are per thread).
"""
import ctypes
import os
import queue
import threading
import time
from concurrent.futures import Future

import numpy as np

from . import drivers as D
from . import graph as G

_LIB = None


def _lib():
    global _LIB
    if _LIB is None:
        lib = ctypes.CDLL(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                       "libmagnet_b200.so"))
        lib.mg_set_stream.argtypes = [ctypes.c_void_p]
        lib.mg_smooth_knn.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                      ctypes.c_int, ctypes.c_void_p]
        lib.mg_last_error.restype = ctypes.c_char_p
        P_, I64 = ctypes.c_void_p, ctypes.c_int64
        lib.mg_knn_search.argtypes = [P_, I64, ctypes.c_int, P_, P_, I64, P_, I64, P_, I64, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_uint64, ctypes.c_int, P_, P_]
        lib.mg_transform_schedule.argtypes = [P_, P_, I64, ctypes.c_int, I64, ctypes.c_double, ctypes.c_int, P_, P_,
                                              P_, ctypes.POINTER(I64)]
        _LIB = lib
    return _LIB


# ----------------------------------------------------------------------------------------------- scheduler
class _Request:
    __slots__ = ("kind", "payload", "nbytes", "points", "future", "t_submit", "t_start", "t_done")

    def __init__(self, kind, payload, nbytes, points):
        self.kind, self.payload, self.nbytes, self.points = kind, payload, int(nbytes), int(points)
        self.future = Future()
        self.t_submit = time.perf_counter()
        self.t_start = self.t_done = None


class Server:
    """FIFO of requests, `slots` workers, admission of each request's device bytes against `budget_bytes`.

    work(kind, payload, slot) -> result runs in the worker thread of `slot`; init(slot) runs once in each worker
    before its first request (e.g. to bind a CUDA stream). Futures carry the result; each request records its
    submit / start / done times (perf_counter seconds)."""

    def __init__(self, work, slots=4, budget_bytes=None, init=None):
        if slots < 1:
            raise ValueError("slots must be at least 1")
        self.work, self.slots, self.budget = work, int(slots), budget_bytes
        self._q = queue.Queue()
        self._cv = threading.Condition()
        self._reserved = 0
        self._tickets = 0            # admission tickets, taken in the order requests leave the FIFO
        self._turn = 0               # the ticket allowed to reserve next
        self.done = []
        self._done_lock = threading.Lock()
        self.peak_reserved = 0
        self._healthy = self.slots   # slots whose start-up succeeded (or has not failed yet)
        self._threads = [threading.Thread(target=self._run, args=(s, init), daemon=True) for s in range(self.slots)]
        for t in self._threads:
            t.start()

    def submit(self, kind, payload, nbytes=0, points=0):
        """queue a request of `nbytes` device bytes over `points` rows; returns its Future"""
        if self.budget is not None and nbytes > self.budget:
            raise ValueError("request needs %d device bytes, more than the server's budget %d" % (nbytes, self.budget))
        r = _Request(kind, payload, nbytes, points)
        self._q.put(r)
        return r.future

    def _admit(self, r):
        # requests reserve in ticket order, so a large request that waits for memory is not overtaken by later
        # small ones; it starts as soon as running requests have released enough
        with self._cv:
            ticket = self._tickets
            self._tickets += 1
            while ticket != self._turn or (self.budget is not None and self._reserved + r.nbytes > self.budget):
                self._cv.wait()
            self._reserved += r.nbytes
            self.peak_reserved = max(self.peak_reserved, self._reserved)
            self._turn += 1
            self._cv.notify_all()

    def _release(self, r):
        with self._cv:
            self._reserved -= r.nbytes
            self._cv.notify_all()

    def _run(self, slot, init):
        init_error = None
        if init is not None:
            try:
                init(slot)
            except BaseException as e:
                init_error = e
            with self._cv:
                if init_error is not None:
                    self._healthy -= 1
                    # a slot that cannot start leaves the work to the others; the last one left fails the
                    # requests instead of letting them wait forever
                    if self._healthy > 0:
                        return
        while True:
            r = self._q.get()
            if r is None:
                return
            self._admit(r)
            r.t_start = time.perf_counter()
            try:
                if init_error is not None:
                    raise RuntimeError("server slot %d failed to start: %s" % (slot, init_error))
                res = self.work(r.kind, r.payload, slot)
                r.t_done = time.perf_counter()
                r.future.set_result(res)
            except BaseException as e:   # the request fails, the server keeps serving
                r.t_done = time.perf_counter()
                r.future.set_exception(e)
            finally:
                self._release(r)
                with self._done_lock:
                    self.done.append(r)

    def close(self):
        for _ in self._threads:
            self._q.put(None)
        for t in self._threads:
            t.join()


def latency_summary(requests, kind=None):
    """p50 / p99 / mean latency (ms, submit to done) and points/s over the requests of one kind"""
    rs = [r for r in requests if kind is None or r.kind == kind]
    if not rs:
        return {}
    lat = np.array([(r.t_done - r.t_submit) * 1e3 for r in rs])
    pts = sum(r.points for r in rs)
    span = max(r.t_done for r in rs) - min(r.t_submit for r in rs)
    return {"requests": len(rs), "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "points_per_s": float(pts / max(span, 1e-9))}


# ----------------------------------------------------------------------------------------------- device work
class FittedLayout:
    """A fitted layout resident on the device: training rows X (n, d), layout Y (n, 2), kernel constants."""

    def __init__(self, X, Y, *, a, b, rep_a=None, rep_b=1.0, n_neighbors=15, transform_epochs=100,
                 learning_rate=1.0, samples_per_node=5.0, parallel="owner", seed=0, query_block=1024,
                 owner_chunk_edges=256, graph=None, landmarks=None, ef=None, n_entry=5):
        import torch
        self.torch = torch
        self.dev = torch.device("cuda", torch.cuda.current_device())
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.ascontiguousarray(Y, dtype=np.float32)
        self.n, self.d = X.shape
        self.Xd = torch.from_numpy(X).to(self.dev)
        self.sq = (self.Xd * self.Xd).sum(1)
        self.Yd = torch.from_numpy(Y).to(self.dev)
        self.a, self.b = float(a), float(b)
        self.rep_a = self.a if rep_a is None else float(rep_a)
        self.rep_b = float(rep_b)
        self.k = min(int(n_neighbors), self.n) - 1
        self.n_neighbors = int(n_neighbors)
        self.epochs = int(transform_epochs)
        self.samples_per_node = float(samples_per_node)
        self.parallel = {"owner": 1, "hogwild": 0}[parallel]
        self.seed = int(seed)
        self.block = int(query_block)
        self.chunk_edges = int(owner_chunk_edges)
        # column tiles of the two-stage top-k: a divisor of n in [1024, 8192] when there is one, else 4096 with
        # the last tile padded
        divisors = [t for t in range(8192, 1023, -1) if self.n % t == 0]
        self.tile = divisors[0] if divisors else min(4096, self.n)
        self.n_tiles = -(-self.n // self.tile)
        # the beam search of magnet/knn.py:131-152 over the training graph, from the landmarks of
        # choose_landmarks(n, random_state) (magnet/knn.py:125-128), ef = max(64, 2k + 10)
        self.search = graph is not None
        if self.search:
            import scipy.sparse as sp
            Gc = sp.csr_matrix(graph)
            if landmarks is None:
                m_l = int(min(self.n, max(100, 4 * np.sqrt(self.n))))
                landmarks = np.sort(np.random.default_rng(self.seed).choice(self.n, m_l, replace=False))
            self.gptr = torch.from_numpy(Gc.indptr.astype(np.int32)).to(self.dev)
            self.gidx = torch.from_numpy(Gc.indices.astype(np.int32)).to(self.dev)
            self.land = torch.from_numpy(np.ascontiguousarray(landmarks, dtype=np.int32)).to(self.dev)
            self.ef = int(ef) if ef else max(64, 2 * self.k + 10)
            self.n_entry = int(n_entry)
        # the step in units of the layout's own spacing (magnet/__init__.py:899-906): min(1, median 1-NN / 0.14)
        from scipy.spatial import cKDTree
        sub = Y[np.random.default_rng(0).choice(self.n, min(self.n, 5000), replace=False)]
        d1 = float(np.median(cKDTree(Y).query(sub, k=2)[0][:, 1]))
        self.lr = float(learning_rate) * float(min(1.0, d1 / 0.14))

    def request_bytes(self, m):
        """device bytes a transform of m rows holds at its peak: a block of query distances (and its padded copy
        when the tiles do not divide n), the first-stage top-k candidates, the neighbour arrays, the layout copy
        and the SGD's per-edge and per-node scratch"""
        if self.search:
            return 12 * m * self.k + 4 * m * self.d + 64 * m * self.k + 48 * (self.n + m)
        mb = min(m, self.block)
        padded = self.n_tiles * self.tile
        dist_block = 4 * mb * self.n + (4 * mb * padded if padded != self.n else 0)
        candidates = 12 * mb * self.n_tiles * self.k
        return dist_block + candidates + 64 * m * self.k + 48 * (self.n + m)

    def bind_stream(self):
        """give this thread a CUDA stream of its own: torch's current stream for the thread, and the C ABI's"""
        st = self.torch.cuda.Stream(device=self.dev)
        self.torch.cuda.set_stream(st)
        _lib().mg_set_stream(ctypes.c_void_p(st.cuda_stream))
        _THREAD.stream = st
        return st

    def knn(self, Qd):
        """exact k nearest training rows of the query rows (squared euclidean), sorted: (ind, dist) on the device.
        The top-k runs in two stages: the k smallest of every tile of `tile` columns, then the k smallest of those
        candidates; a tile's top-k over a few thousand columns is far cheaper than one over all n."""
        torch = self.torch
        m = Qd.shape[0]
        qs = (Qd * Qd).sum(1)
        ind = torch.empty((m, self.k), dtype=torch.int64, device=self.dev)
        dist = torch.empty((m, self.k), dtype=torch.float32, device=self.dev)
        T, nt = self.tile, self.n_tiles
        for s in range(0, m, self.block):
            q = Qd[s:s + self.block]
            r = q.shape[0]
            # |x|^2 - 2 q.x in one GEMM with bias; the row's |q|^2 does not change its order and is added to the
            # k selected values only
            d2 = torch.addmm(self.sq[None, :].expand(r, self.n), q, self.Xd.T, beta=1.0, alpha=-2.0)
            if nt * T != self.n:
                d2 = torch.cat([d2, torch.full((r, nt * T - self.n), float("inf"), device=self.dev)], 1)
            v1, i1 = torch.topk(d2.view(r, nt, T), self.k, dim=2, largest=False, sorted=False)
            v, j = torch.topk(v1.reshape(r, nt * self.k), self.k, dim=1, largest=False, sorted=True)
            tile_of = torch.div(j, self.k, rounding_mode="floor")
            local = torch.gather(i1.reshape(r, nt * self.k), 1, j)
            ind[s:s + r] = tile_of * T + local
            dist[s:s + r] = torch.sqrt(torch.clamp(v + qs[s:s + r, None], min=0.0))
        return ind, dist

    def beam(self, Qd):
        """the k training rows found by the beam search for the query rows, and their distances (the square roots
        of the squared distances, magnet/knn.py:80-83): (ind, dist) on the device"""
        torch = self.torch
        m = Qd.shape[0]
        ind = torch.empty((m, self.k), dtype=torch.int32, device=self.dev)
        d2 = torch.empty((m, self.k), dtype=torch.float32, device=self.dev)
        rc = _lib().mg_knn_search(ctypes.c_void_p(self.Xd.data_ptr()), self.n, self.d,
                                  ctypes.c_void_p(self.gptr.data_ptr()), ctypes.c_void_p(self.gidx.data_ptr()),
                                  int(self.gidx.numel()), ctypes.c_void_p(self.land.data_ptr()),
                                  int(self.land.numel()), ctypes.c_void_p(Qd.data_ptr()), m, self.k, self.ef,
                                  self.n_entry, self.seed, -1, ctypes.c_void_p(ind.data_ptr()),
                                  ctypes.c_void_p(d2.data_ptr()))
        if rc != 0:
            raise RuntimeError(_lib().mg_last_error().decode())
        return ind.long(), torch.sqrt(torch.clamp(d2, min=0.0))

    def transform(self, X_new, seed=None):
        """new rows (m, d) -> their layout positions (m, 2), on this thread's stream"""
        torch = self.torch
        from . import _native as N
        if len(X_new) == 0:
            return np.zeros((0, self.Yd.shape[1]), np.float32)
        st = getattr(_THREAD, "stream", None)
        if st is None:
            # a thread that is not a server worker: the caller's current stream, for torch and the C ABI alike
            st = torch.cuda.current_stream(self.dev)
            _lib().mg_set_stream(ctypes.c_void_p(st.cuda_stream))
        with torch.cuda.stream(st):
            Q = torch.from_numpy(np.ascontiguousarray(X_new, dtype=np.float32)).to(self.dev, non_blocking=False)
            m = Q.shape[0]
            ind, dist = self.beam(Q) if self.search else self.knn(Q)
            vals = torch.empty_like(dist)
            rc = _lib().mg_smooth_knn(ctypes.c_void_p(dist.data_ptr()), m, self.k, self.n_neighbors, 1.0, 64,
                                      ctypes.c_void_p(vals.data_ptr()))
            if rc != 0:
                raise RuntimeError(_lib().mg_last_error().decode())
            W = vals / torch.clamp(vals.sum(1, keepdim=True), min=1e-12)
            Y_new = torch.einsum("mk,mkd->md", W, self.Yd[ind])
            # the edge schedule of MAGNET.transform (magnet/__init__.py:907-912), on the device
            ind = ind.long().contiguous()
            vals = vals.contiguous()
            n_e = m * self.k
            head = torch.empty(n_e, dtype=torch.int32, device=self.dev)
            tail = torch.empty(n_e, dtype=torch.int32, device=self.dev)
            eps = torch.empty(n_e, dtype=torch.float32, device=self.dev)
            kept = ctypes.c_int64(0)
            rc = _lib().mg_transform_schedule(ctypes.c_void_p(vals.data_ptr()), ctypes.c_void_p(ind.data_ptr()), m,
                                              self.k, self.n, float(self.samples_per_node), self.epochs,
                                              ctypes.c_void_p(head.data_ptr()), ctypes.c_void_p(tail.data_ptr()),
                                              ctypes.c_void_p(eps.data_ptr()), ctypes.byref(kept))
            if rc != 0:
                raise RuntimeError(_lib().mg_last_error().decode())
            head, tail, eps = head[:kept.value], tail[:kept.value], eps[:kept.value]
            Y_all = torch.cat([self.Yd, Y_new.to(torch.float32)]).contiguous()
            eons = eps.clone()
            eonns = (eps / 5.0).contiguous()
            z = torch.zeros(0, dtype=torch.int32, device=self.dev)
            zf = torch.zeros(0, dtype=torch.float32, device=self.dev)
            z2 = torch.zeros((0, 2), dtype=torch.float32, device=self.dev)
            sd = self.seed if seed is None else int(seed)
            N.optimize_layout(Y_all, head, tail, eps, eons, eonns, z, z, 0, self.epochs, self.lr, 0.0, 0.0, 0.0,
                              self.a, self.b, self.rep_a, self.rep_b, 5.0, 0, 1.0, 2.0, 4, 0.25, 0, 0, self.n,
                              z2, z2, z, 0.9, 0.999, z, np.zeros((0, 1), np.int32), z, z, 0.0, 0, zf, sd, -1,
                              self.parallel, None, None, 0, owner_chunk_edges=self.chunk_edges)
            out = Y_all[self.n:].cpu().numpy()
        return out


_THREAD = threading.local()


def fit_layout(X, *, n_neighbors=15, n_epochs=200, a=None, b=None, seed=0, parallel="hogwild",
               return_graph=False):
    """a fit request: exact kNN, the fuzzy graph and the edge schedule, a PCA start rescaled as the reference's
    init, then the sampled SGD with 5 mid-near pairs, all device passes on this thread's stream"""
    if a is None or b is None:
        a, b = D.find_ab_params(1.0, 0.1)
    X = np.ascontiguousarray(X, dtype=np.float32)
    ind, dist = G.exact_knn(X, n_neighbors)
    P = G.fuzzy_graph(ind, dist, n_neighbors)
    head, tail, eps = D.edge_schedule(P, n_epochs, device=True)
    Y = G.initial_layout(G.pca2(X, seed), seed)
    pairs = G.mid_near_pairs(X, 5, 6, seed=seed)
    D.optimize_sgd(Y, head, tail, eps, n_epochs, a=a, b=b, mid_weight=0.1, mid_pairs=pairs, graph=P, seed=seed,
                   parallel=parallel)
    return (Y, P) if return_graph else Y


def device_server(layout, slots=4, budget_fraction=0.5):
    """a Server whose workers run transform ("transform", X_new[, seed]) and fit ("fit", X) requests, each
    worker on its own CUDA stream; the memory budget is a fraction of the device's free bytes"""
    free, _ = layout.torch.cuda.mem_get_info()

    def init(slot):
        layout.torch.cuda.set_device(layout.dev)
        layout.bind_stream()

    def work(kind, payload, slot):
        if kind == "transform":
            X_new, seed = payload if isinstance(payload, tuple) else (payload, None)
            return layout.transform(X_new, seed)
        if kind == "fit":
            return fit_layout(payload)
        raise ValueError("unknown request kind " + str(kind))

    return Server(work, slots=slots, budget_bytes=int(free * budget_fraction), init=init)


def fit_bytes(m, d, n_neighbors=15):
    """device bytes a fit of m rows holds at its peak (a block of 2048 distance rows, the graph and SGD)"""
    return 4 * min(m, 2048) * m + 4 * m * d + 200 * m * n_neighbors
