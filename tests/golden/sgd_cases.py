"""optimize_layout option cases beyond the defaults, on the sgd_small.npz inputs (600 points, 5 blobs, kNN
graph of 15, 40 epochs). Each case is the full keyword set of the reference's binding (src/bindings.cpp:11-23)
except the eight positional arrays, so one dict drives the reference's `_magnet.optimize_layout`, the oracle's
`sgd_serial` and the device's `optimize_layout`. Options follow the reference's driver (magnet/__init__.py:755-803):
loss 0 umap / 1 InfoNCE, kernel 0 power / 1 gaussian / 2 sech / 3 tanh, optimizer 1 = per-node lazy Adam with
zero state (also with n_fixed), clip_mode 1 = step-norm cap, a jump graph over the mid-near pairs, per-node walk
lengths and b, rep_b <= 0 for the coupled repulsion kernel, and dims other than 2. Pure numpy: the tests import it
without the reference."""
import numpy as np

CASES = ["infonce", "gaussian", "sech", "tanh", "adam", "adam_n_fixed", "norm_clip", "jump", "walk_lens",
         "node_b", "coupled", "exaggeration", "dim3", "dim8_walk"]

# cases whose draws the device records through the schedule hook (the mid partner, walk and jump draws)
SCHEDULE_CASES = ["infonce", "jump", "walk_lens", "dim3"]


def _jump_graph(mid_pairs):
    """CSR of the mid-near pairs (row i -> its partners), the jump graph of the reference's driver"""
    n, m = mid_pairs.shape
    indptr = np.arange(0, n * m + 1, m, dtype=np.int32)
    return indptr, np.ascontiguousarray(mid_pairs.reshape(-1), dtype=np.int32)


def _initial(g, dim):
    n = g["Y0"].shape[0]
    return g["Y0"].copy() if dim == 2 else np.random.default_rng(dim).uniform(-10, 10, (n, dim)).astype(np.float32)


def _base_kw(g, dim, seed):
    """the default options: umap loss, power kernel a = 1.7, b = 0.8, sgd, coordinate clip, 5 mid-near pairs"""
    z = np.zeros(0, np.int32)
    return dict(indptr=z, indices=z, epoch_start=0, epoch_end=40, alpha0=1.0, alpha1=0.0, mid_w0=0.1, mid_w1=0.0,
                a=1.7, b=0.8, rep_a=1.7382, rep_b=1.0, negative_sample_rate=5.0, loss=0, exaggeration=1.0,
                repulsion_strength=2.0, walk_len=4, mid_rate=0.25, optimizer=0, clip_mode=0, n_fixed=0,
                adam_m=np.zeros((0, dim), np.float32), adam_v=np.zeros((0, dim), np.float32), adam_t=z,
                beta1=0.9, beta2=0.999, walk_lens=z, mid_pairs=g["mid_pairs"], jump_indptr=z, jump_indices=z,
                mid_jump=0.0, kernel=0, node_b=np.zeros(0, np.float32), seed=seed)


def _adam_state(kw, n, dim):
    kw.update(optimizer=1, adam_m=np.zeros((n, dim), np.float32), adam_v=np.zeros((n, dim), np.float32),
              adam_t=np.zeros(n, np.int32), beta1=0.8, beta2=0.99)


def state(g, name, seed=12345):
    """(Y, eons, eonns, kwargs) for one case, fresh arrays every call"""
    n = g["Y0"].shape[0]
    eps = g["eps"]
    dim = {"dim3": 3, "dim8_walk": 8}.get(name, 2)
    Y = _initial(g, dim)
    kw = _base_kw(g, dim, seed)
    if name == "infonce":
        kw.update(loss=1)
    elif name in ("gaussian", "sech", "tanh"):
        kw.update(kernel={"gaussian": 1, "sech": 2, "tanh": 3}[name])
    elif name in ("adam", "adam_n_fixed"):
        # Adam's steps stay below the 4 alpha cap (|m/c1| / sqrt(v/c2) is about 1), so the clip mode never acts on
        # them; the second case holds the first 200 nodes fixed (the transform setting)
        _adam_state(kw, n, dim)
        kw.update(n_fixed=200 if name == "adam_n_fixed" else 0)
    elif name == "norm_clip":
        kw.update(clip_mode=1)
    elif name == "jump":
        jp, jx = _jump_graph(g["mid_pairs"])
        kw.update(indptr=g["indptr"], indices=g["indices"], jump_indptr=jp, jump_indices=jx, mid_jump=0.5)
    elif name == "walk_lens":
        kw.update(indptr=g["indptr"], indices=g["indices"], mid_pairs=np.zeros((0, 1), np.int32),
                  walk_lens=np.random.default_rng(7).integers(0, 9, n).astype(np.int32))
    elif name == "node_b":
        kw.update(node_b=np.random.default_rng(8).uniform(0.5, 1.5, n).astype(np.float32))
    elif name == "coupled":
        kw.update(rep_b=0.0)
    elif name == "exaggeration":
        kw.update(exaggeration=4.0, repulsion_strength=1.0, negative_sample_rate=3.0, mid_rate=0.5)
    elif name == "dim8_walk":
        kw.update(indptr=g["indptr"], indices=g["indices"], mid_pairs=np.zeros((0, 1), np.int32), walk_len=3)
    elif name != "dim3":
        raise KeyError(name)
    eons = eps.copy()
    eonns = (eps / kw["negative_sample_rate"]).astype(np.float32)
    return Y, eons, eonns, kw


def oracle_kw(kw):
    """the same case as keywords of the oracle's argument builder (empty arrays become None)"""
    out = {}
    for k, v in kw.items():
        if isinstance(v, np.ndarray) and v.size == 0:
            continue
        out[k] = v
    return out


def purity(Y, labels, k=10):
    """fraction of each point's k nearest neighbours in the layout that share its blob label"""
    from sklearn.neighbors import NearestNeighbors
    nn = NearestNeighbors(n_neighbors=k + 1).fit(Y).kneighbors(Y, return_distance=False)[:, 1:]
    return float((labels[nn] == labels[:, None]).mean())


def expected(g, opts, name):
    """the reference's final (Y, eons, eonns) for a case: sgd_options.npz, whose bookkeeping arrays are stored only
    where they differ from the default run's in sgd_small.npz"""
    return (opts[f"Y_{name}"], opts.get(f"eons_{name}", g["eons_default"]),
            opts.get(f"eonns_{name}", g["eonns_default"]))


# ---------------------------------------------------------------------------------------------- owner mode
# parallel = 1 (src/layout.cpp:441-463): chunks of about 4096 edges, one stream per chunk, reads from the layout at
# the start of the epoch. The "_b1" cases use only +, *, / and sqrt (power kernel with b = rep_b = 1, the sgd
# optimizer), which the device evaluates as the reference's plain x86-64 build does; the others go through powf,
# expf or tanhf. "large" is an 8000-node graph (23 chunks); "dup" starts from 16 distinct positions, so that
# negatives at distance 0 draw the jitter (with Adam, the replay also restores the Adam state).
OWNER_CASES = ["b1_pairs", "b1_walk_fixed", "b1_jump_norm_dim3", "b1_dim8", "b1_large", "b1_dup", "pairs",
               "adam_b1", "adam_b1_dup", "node_b", "gaussian_large"]


def synthetic_graph(n=8000, k=12, centers=8, seed=3):
    """a blob-structured graph with rows sorted by head: k same-blob neighbours per node, epochs_per_sample from
    uniform weights, 5 random mid-near pairs per node"""
    rng = np.random.default_rng(seed)
    labels = rng.integers(0, centers, n)
    members = [np.flatnonzero(labels == c) for c in range(centers)]
    tail = np.empty(n * k, np.int32)
    for i in range(n):
        cand = rng.choice(members[labels[i]], k + 1, replace=False)
        tail[i * k:(i + 1) * k] = cand[cand != i][:k]
    w = rng.uniform(0.05, 1.0, n * k)
    eps = (w.max() / w).astype(np.float32)
    return dict(Y0=rng.uniform(-10, 10, (n, 2)).astype(np.float32), head=np.repeat(np.arange(n, dtype=np.int32), k),
                tail=tail, eps=eps, indptr=np.arange(0, n * k + 1, k, dtype=np.int32), indices=tail.copy(),
                mid_pairs=rng.integers(0, n, (n, 5)).astype(np.int32), labels=labels)


def reverse_pairs(mid_pairs, n):
    """who chose each node as a mid-range partner, CSR (the reference's driver, magnet/__init__.py:789-794)"""
    import scipy.sparse as sp
    m = mid_pairs.shape[1]
    R = sp.csr_matrix((np.ones(mid_pairs.size, np.float32), (mid_pairs.ravel(), np.repeat(np.arange(n), m))),
                      shape=(n, n))
    R.sort_indices()
    return R.indptr.astype(np.int32), R.indices.astype(np.int32)


def owner_state(g, name, seed=12345, big=None):
    """(inputs, Y, eons, eonns, kwargs, rev_indptr, rev_indices) of an owner case; kwargs exclude parallel and the
    reverse pairs, which are built from the mid-near pairs as the reference's driver does. `big` caches
    synthetic_graph() for the "_large" cases."""
    if name.endswith("_large"):
        g = big if big is not None else synthetic_graph()
    n = g["Y0"].shape[0]
    dim = {"b1_jump_norm_dim3": 3, "b1_dim8": 8}.get(name, 2)
    Y = _initial(g, dim)
    if name.endswith("_dup"):
        Y = np.random.default_rng(4).uniform(-10, 10, (16, 2)).astype(np.float32)[np.arange(n) % 16]
    kw = _base_kw(g, dim, seed)
    if name.startswith("b1") or name.startswith("adam_b1"):
        kw.update(b=1.0, rep_a=1.7, rep_b=1.0)
    if name.startswith("adam_b1"):
        _adam_state(kw, n, dim)
    elif name == "b1_walk_fixed":
        kw.update(indptr=g["indptr"], indices=g["indices"], mid_pairs=np.zeros((0, 1), np.int32), n_fixed=100)
    elif name == "b1_jump_norm_dim3":
        jp, jx = _jump_graph(g["mid_pairs"])
        kw.update(indptr=g["indptr"], indices=g["indices"], jump_indptr=jp, jump_indices=jx, mid_jump=0.5,
                  walk_lens=np.random.default_rng(7).integers(0, 9, n).astype(np.int32), clip_mode=1)
    elif name == "node_b":
        kw.update(node_b=np.random.default_rng(8).uniform(0.5, 1.5, n).astype(np.float32))
    elif name == "gaussian_large":
        kw.update(kernel=1)
    rp = rx = np.zeros(0, np.int32)
    if kw["mid_pairs"].size > 0 and kw["jump_indptr"].size == 0:
        rp, rx = reverse_pairs(kw["mid_pairs"], n)
    eons = g["eps"].copy()
    eonns = (g["eps"] / kw["negative_sample_rate"]).astype(np.float32)
    return g, Y, eons, eonns, kw, rp, rx


def digest(a):
    """sha-256 of an array's bytes (C order), the compact form of bit-exact bookkeeping in the fixtures"""
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


# settings of the kernel fit find_ab_params (magnet/__init__.py:26-48): the default, a given b (the bench's
# size-dependent b), another spread, and the gaussian, sech and tanh kernels
AB_CASES = [dict(spread=1.0, min_dist=0.1), dict(spread=1.0, min_dist=0.05, b=0.6),
            dict(spread=1.5, min_dist=0.2), dict(spread=1.0, min_dist=0.1, kernel="gaussian"),
            dict(spread=1.0, min_dist=0.1, kernel="sech"), dict(spread=1.0, min_dist=0.1, kernel="tanh")]
