"""The drop-in, shown by replay: every call that the reference's own estimator (magnet/__init__.py:496-930,
MAGNET.fit_transform with loss "umap", "tsne" and "hybrid", and MAGNET.transform) made into its native module
`_magnet` is made again, with the same positional and keyword arguments, into this repository's `_magnet`
(lib-magnet_b200/_magnet), and each result is compared with the one the reference's module returned.

The calls were recorded by running the reference's estimator unchanged on top of a recording stand-in for its
`_magnet` (tests/golden/make_dropin_golden.py): its Python package cannot travel to the GPU machine, so the
estimator itself cannot run there. The layout-pass entry points, the mid-near partners, the query search and the
spectral solver run on the device; NN-descent is forwarded to the reference's compiled module (oracle/_ref)
through MAGNET_HOST_MODULE, as the drop-in is meant to be installed.

Bounds per entry point (the same as the entry points' own tests): bbox_2d exact; tsne_attraction, tsne_step,
tsne_update, mid_spring and smooth_knn within 1e-5 relative; FFTConv2D.compute's sumQ and F within 1e-4 relative;
chebyshev_eigenvectors' leading Ritz vectors spanning the reference's subspace (largest principal-angle sine 1e-3);
optimize_layout's schedule state (epoch_of_next_sample, epoch_of_next_negative_sample) bit-exact, its layout (the
device's own random streams) finite and moved by as much as the reference's within a factor of 2.
"""
import glob
import importlib.util
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def shim(mg):
    host = glob.glob(os.path.join(ROOT, "oracle", "_ref", "_magnet*.so"))
    if not host:
        pytest.skip("the reference module (oracle/_ref) is not built")
    os.environ["MAGNET_HOST_MODULE"] = host[0]
    spec = importlib.util.spec_from_file_location("_magnet_dropin_under_test",
                                                  os.path.join(ROOT, "lib-magnet_b200", "_magnet", "__init__.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="module")
def recording(golden):
    g = golden("dropin_calls.npz")
    meta = json.loads(bytes(g["meta"]).decode())
    return g, meta


def decode(g, v):
    if "array" in v:
        return np.array(g[v["array"]], copy=True)
    if "tuple" in v:
        return tuple(decode(g, x) for x in v["tuple"])
    return v["value"]


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def subspace_sine(A, B):
    """the largest sine of the principal angles between the column spans of A and B"""
    qa, _ = np.linalg.qr(A)
    qb, _ = np.linalg.qr(B)
    cos = np.clip(np.linalg.svd(qa.T @ qb, compute_uv=False), 0.0, 1.0)
    return float(np.sqrt(max(0.0, 1.0 - cos.min() ** 2)))


def check_call(g, c, args, out):
    name = c["name"]
    ret = decode(g, c["ret"])
    inplace = {int(k): decode(g, v) for k, v in c["inplace"].items()}
    if name == "bbox_2d":
        assert tuple(np.float32(x) for x in out) == tuple(np.float32(x) for x in ret)
    elif name in ("tsne_attraction", "smooth_knn"):
        out = np.asarray(out)
        assert out.shape == ret.shape
        assert np.allclose(out, ret, rtol=1e-5, atol=1e-5 * np.abs(ret).max()), rel(out, ret)
    elif name == "FFTConv2D.compute":
        sq, F = out
        assert abs(sq - ret[0]) / abs(ret[0]) < 1e-4, (sq, ret[0])
        assert rel(F, ret[1]) < 1e-4
    elif name in ("tsne_step", "tsne_update", "mid_spring"):
        for i, want in inplace.items():
            assert np.allclose(args[i], want, rtol=1e-5, atol=1e-5 * max(np.abs(want).max(), 1e-30)), \
                (name, i, rel(args[i], want))
    elif name == "optimize_layout":
        assert np.array_equal(args[4], inplace[4]) and np.array_equal(args[5], inplace[5])
        assert np.isfinite(args[0]).all()
        return args[0]
    elif name in ("mid_near_pairs_dense", "knn_search"):
        o, r = (out, ret) if name == "mid_near_pairs_dense" else (out[0], ret[0])
        assert np.array_equal(np.asarray(o), np.asarray(r))   # the device reproduces the reference's streams
    elif name == "chebyshev_eigenvectors":
        # on the device now: the leading n_wanted Ritz vectors span the reference's subspace
        o, r = np.asarray(out, np.float64), np.asarray(ret, np.float64)
        nw = int(args[6])
        assert o.shape == r.shape and np.isfinite(o).all()
        assert subspace_sine(o[:, :nw], r[:, :nw]) < 1e-3, subspace_sine(o[:, :nw], r[:, :nw])
    elif name == "nn_descent":
        o = out[0] if isinstance(out, tuple) else out
        r = ret[0] if isinstance(ret, tuple) else ret
        assert np.asarray(o).shape == np.asarray(r).shape     # forwarded; multithreaded on the host
    return None


def test_estimator_calls_replay_through_dropin(mg, shim, recording):
    g, meta = recording
    calls = meta["calls"]
    objs = {}
    seen = {}
    l0 = mg.launch_count()
    moved = []
    for c in calls:
        name = c["name"]
        args = [decode(g, a) for a in c["args"]]
        kwargs = {k: decode(g, v) for k, v in c["kwargs"].items()}
        if name == "FFTConv2D":
            objs[c["obj"]] = shim.FFTConv2D(*args, **kwargs)
            out = None
        elif name.startswith("FFTConv2D."):
            out = getattr(objs[c["obj"]], name.split(".", 1)[1])(*args, **kwargs)
        else:
            y_in = args[0].copy() if name == "optimize_layout" else None
            out = getattr(shim, name)(*args, **kwargs)
            if name == "optimize_layout":
                y_ref = decode(g, c["inplace"]["0"])
                moved.append((np.sqrt(((args[0] - y_in) ** 2).sum(1).mean()),
                              np.sqrt(((y_ref - y_in) ** 2).sum(1).mean())))
        check_call(g, c, args, out)
        seen[name] = seen.get(name, 0) + 1
    launches = mg.launch_count() - l0
    print("replayed %d calls: %s; %d device kernels" % (len(calls), seen, launches))
    for d, r in moved:
        assert 0.5 * r <= d <= 2.0 * r, (d, r)
    for name in ("optimize_layout", "tsne_attraction", "bbox_2d", "FFTConv2D.compute", "tsne_step", "tsne_update",
                 "mid_spring", "smooth_knn"):
        assert seen.get(name, 0) > 0, name
    assert launches > 0
