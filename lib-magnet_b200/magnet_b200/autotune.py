"""Launch-shape autotuner of the batched t-SNE form, with a JSON cache keyed by the batch's shape.

What it chooses, by timing a few iterations of the batch itself on the device:
  * threads per row of the attraction (the lanes that share one point's affinity row: 1-32);
  * branches: how many of the batch's layouts run side by side in the iteration graph.
What it leaves alone: the interpolation grid (box count and width). The reference chooses the box count from the
layout's extent (box width 0.7, 20-1000 boxes, magnet/tsne.py:30-46) and that choice defines the result, so the
batch keeps it; each layout's grid allocation is sized from its point count (64 + 2 ceil(sqrt(n)) boxes).

The cache lives in $MAGNET_B200_CACHE (a directory), else ~/.cache/magnet_b200; its key is the layout count, the
median size and the mean row length of the affinities, each rounded to a power of two, and the device name.
"""
import json
import os
import time

import numpy as np

TPR = (2, 4, 8, 16)
BRANCHES = (8, 16, 32, 64)


def cache_path():
    root = os.environ.get("MAGNET_B200_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "magnet_b200")
    return os.path.join(root, "autotune.json")


def _load():
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(table):
    path = cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + ".%d.tmp" % os.getpid()
        with open(tmp, "w") as f:
            json.dump(table, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass   # a read-only home: the choice is still returned, only not kept


def batch_key(sizes, nnzs):
    import torch
    sizes = np.asarray(sizes, dtype=np.float64)
    deg = float(np.sum(nnzs)) / max(float(sizes.sum()), 1.0)
    p2 = lambda x: int(round(np.log2(max(x, 1.0))))
    name = torch.cuda.get_device_name() if torch.cuda.is_available() else "cpu"
    return "tsne_batch|count=%d|n=2^%d|deg=2^%d|%s" % (len(sizes), p2(np.median(sizes)), p2(deg), name)


def lookup(key):
    return _load().get(key)


def tune_tsne_batch(graphs, Ys, params, iters=20, tpr=TPR, branches=BRANCHES, key=None):
    """times `iters` iterations of the batch for each threads-per-row value (at the middle branch count), then each
    branch count at the best of those; returns {"threads_per_row": t, "branches": b, "ms": {...}} and caches it under
    `key` (batch_key of the sizes when None)"""
    from . import _native as N
    if key is None:
        key = batch_key([g[0].size - 1 for g in graphs], [g[1].size for g in graphs])

    def timed(t, b):
        batch = N.TsneBatch(graphs, n_iter=iters, threads_per_row=t, branches=b, **params)
        batch.run([y.copy() for y in Ys])             # capture + warm-up
        Y = [y.copy() for y in Ys]
        t0 = time.perf_counter()
        batch.run(Y)
        return (time.perf_counter() - t0) * 1e3
    ms = {}
    mid = branches[len(branches) // 2]
    for t in tpr:
        ms["tpr=%d,branches=%d" % (t, mid)] = timed(t, mid)
    best_t = min(tpr, key=lambda t: ms["tpr=%d,branches=%d" % (t, mid)])
    for b in branches:
        k = "tpr=%d,branches=%d" % (best_t, b)
        if k not in ms:
            ms[k] = timed(best_t, b)
    best_b = min(branches, key=lambda b: ms["tpr=%d,branches=%d" % (best_t, b)])
    choice = {"threads_per_row": int(best_t), "branches": int(best_b), "ms": {k: round(v, 3) for k, v in ms.items()},
              "iters": int(iters)}
    table = _load()
    table[key] = choice
    _store(table)
    return choice
