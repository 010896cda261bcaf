"""Generates tests/golden/dropin_calls.npz: every call that the reference's own estimator makes into its native
module `_magnet`, with arguments and results, for the drop-in replay test (tests/test_gpu_dropin.py).

The reference's Python package (magnet/) cannot travel to a machine without the reference checkout, so its
estimator cannot run on top of the device module there. Instead it runs here, unchanged, on top of a recording
stand-in for `_magnet` that forwards every call to the reference's compiled module (oracle/_ref) and records the
call's name, its positional and keyword arguments and its results (return values, and the arrays it updates in
place). The scenarios, on 300 points (4 Gaussians in d = 10, seed 7) and 40 new rows:
  * MAGNET(loss="umap", n_epochs=30, random_state=0).fit_transform(X), then .transform(X_new);
  * MAGNET(loss="tsne", n_epochs=20, random_state=0).fit_transform(X) (the mid-range spring path:
    tsne_attraction, bbox_2d, FFTConv2D, mid_spring, tsne_update);
  * MAGNET(loss="hybrid", n_epochs=30, hybrid_iter=10, random_state=0).fit_transform(X) (optimize_layout, then
    the fused path: tsne_attraction, bbox_2d, FFTConv2D, tsne_step).
Arrays are stored once per distinct content.

Runs only where the reference checkout is available (MAGNET_REFERENCE_DIR, else the folder `reference` beside
this repository) and its native module has been compiled by oracle/build_ref.sh.

    python tests/golden/make_dropin_golden.py
"""
import hashlib
import json
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("MAGNET_REFERENCE_DIR", os.path.join(os.path.dirname(ROOT), "reference"))
sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))
import _magnet as _real  # noqa: E402  (the reference's compiled module)

ARRAYS = {}
CALLS = []


def _store(a):
    a = np.ascontiguousarray(a)
    h = hashlib.sha1(a.tobytes() + str((a.dtype, a.shape)).encode()).hexdigest()[:16]
    ARRAYS.setdefault("a_" + h, a.copy())
    return {"array": "a_" + h}


def _enc(v):
    if isinstance(v, np.ndarray):
        return _store(v)
    if isinstance(v, (tuple, list)):
        return {"tuple": [_enc(x) for x in v]}
    if isinstance(v, (np.floating, float)):
        return {"value": float(v)}
    if isinstance(v, (np.integer, int, bool)):
        return {"value": int(v)}
    if v is None:
        return {"value": None}
    raise TypeError(type(v))


# functions that update arrays in place: positional indices of the updated arguments
IN_PLACE = {"optimize_layout": (0, 4, 5, 27, 28, 29), "tsne_step": (0, 1, 2), "tsne_update": (0, 1, 2),
            "mid_spring": (2,)}


def _recorder(name):
    fn = getattr(_real, name)

    def call(*args, **kwargs):
        rec = {"name": name, "args": [_enc(a) for a in args], "kwargs": {k: _enc(v) for k, v in kwargs.items()}}
        out = fn(*args, **kwargs)
        rec["ret"] = _enc(out if not isinstance(out, np.ndarray) else np.asarray(out))
        rec["inplace"] = {str(i): _enc(args[i]) for i in IN_PLACE.get(name, ()) if i < len(args)
                          and isinstance(args[i], np.ndarray) and args[i].size}
        CALLS.append(rec)
        return out
    return call


class FFTConv2D:
    """recording stand-in of the reference's FFTConv2D class"""
    _count = 0

    def __init__(self, M, n_interp):
        FFTConv2D._count += 1
        self.id = FFTConv2D._count
        self.obj = _real.FFTConv2D(M, n_interp)
        CALLS.append({"name": "FFTConv2D", "obj": self.id, "args": [_enc(int(M)), _enc(int(n_interp))],
                      "kwargs": {}, "ret": {"value": None}, "inplace": {}})

    def set_kernels(self, K1h, K2h):
        CALLS.append({"name": "FFTConv2D.set_kernels", "obj": self.id, "args": [_enc(K1h), _enc(K2h)],
                      "kwargs": {}, "ret": {"value": None}, "inplace": {}})
        return self.obj.set_kernels(K1h, K2h)

    def compute(self, *args, **kwargs):
        rec = {"name": "FFTConv2D.compute", "obj": self.id, "args": [_enc(a) for a in args],
               "kwargs": {k: _enc(v) for k, v in kwargs.items()}, "inplace": {}}
        out = self.obj.compute(*args, **kwargs)
        rec["ret"] = _enc((float(out[0]), np.asarray(out[1])))
        CALLS.append(rec)
        return out


def install():
    mod = types.ModuleType("_magnet")
    mod.FFTConv2D = FFTConv2D
    mod.__getattr__ = lambda name: _recorder(name)
    sys.modules["_magnet"] = mod


def blobs(n, d, centers, seed):
    rng = np.random.default_rng(seed)
    C = rng.normal(0, 6, (centers, d))
    y = rng.integers(0, centers, n)
    return (C[y] + rng.normal(0, 1, (n, d))).astype(np.float32), y


def main():
    install()
    sys.path.insert(0, REF)
    from magnet import MAGNET
    X, y = blobs(340, 10, 4, seed=7)
    X, Xnew = X[:300], X[300:]
    scenes = []

    def scene(label, fn):
        start = len(CALLS)
        Y = fn()
        scenes.append({"label": label, "first": start, "end": len(CALLS), "result": _enc(np.asarray(Y))})

    est = MAGNET(loss="umap", n_epochs=30, random_state=0)
    scene("umap fit_transform", lambda: est.fit_transform(X))
    scene("umap transform", lambda: est.transform(Xnew))
    scene("tsne fit_transform", lambda: MAGNET(loss="tsne", n_epochs=20, random_state=0).fit_transform(X))
    scene("hybrid fit_transform",
          lambda: MAGNET(loss="hybrid", n_epochs=30, hybrid_iter=10, random_state=0).fit_transform(X))
    meta = {"calls": CALLS, "scenes": scenes}
    np.savez_compressed(os.path.join(HERE, "dropin_calls.npz"), meta=np.frombuffer(json.dumps(meta).encode(), np.uint8),
                        X=X, Xnew=Xnew, labels=y, **ARRAYS)
    names = {}
    for c in CALLS:
        names[c["name"]] = names.get(c["name"], 0) + 1
    print(len(CALLS), "calls,", len(ARRAYS), "arrays:", names)


if __name__ == "__main__":
    main()
