"""SGD layout on the device against the reference. The schedule (which edges are sampled, how many negatives)
and the negative-sample indices match bit-exactly: the serial stream mode against the reference's single
stream per epoch (n_threads = 1), the per-edge stream mode against the oracle's replay of the same streams. The
eons / eonns bookkeeping after a whole run equals the reference's bit-for-bit; layouts match in quality."""
import numpy as np
import pytest

import sgd_cases as C
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def sched_kw(g, mid=True):
    kw = dict(a=1.7, b=0.8, rep_a=1.7382, seed=12345, epoch_start=0, epoch_end=40, alpha0=1.0, alpha1=0.0)
    if mid:
        kw.update(mid_pairs=g["mid_pairs"], mid_w0=0.1, mid_w1=0.0)
    return kw


@pytest.mark.parametrize("stream_mode", [1, 0])
@pytest.mark.parametrize("mid", [True, False])
def test_schedule_and_negatives_bit_exact(mg, golden, stream_mode, mid):
    g = golden("sgd_small.npz")
    eps = g["eps"]
    e_o, en_o = eps.copy(), (eps / 5).astype(np.float32)
    e_d, en_d = eps.copy(), (eps / 5).astype(np.float32)
    kw = sched_kw(g, mid)
    for epoch in range(6):
        s_o, n_o, off_o, negs_o, mid_o = O.sgd_schedule(g["Y0"].copy(), g["head"], g["tail"], eps, e_o, en_o,
                                                        epoch, per_edge_stream=(stream_mode == 0), **kw)
        s_d, n_d, off_d, negs_d, mid_d = mg.layout_schedule(
            g["Y0"].copy(), g["head"], g["tail"], eps, e_d, en_d, epoch, 0, 40, 1.0, 0.0,
            kw.get("mid_w0", 0.0), kw.get("mid_w1", 0.0), mid_pairs=kw.get("mid_pairs"), seed=12345,
            stream_mode=stream_mode)
        assert np.array_equal(s_o.astype(bool), s_d.astype(bool))
        assert np.array_equal(n_o, n_d)
        assert np.array_equal(negs_o, negs_d)
        assert np.array_equal(mid_o, mid_d)
        assert np.array_equal(e_o, e_d) and np.array_equal(en_o, en_d)


def run_layout(mg, g, stream_mode, case="default", seed=12345):
    Y = g["Y0"].copy(); eps = g["eps"]; eons = eps.copy(); eonns = (eps / 5).astype(np.float32)
    z = np.zeros(0, np.int32)
    mp = g["mid_pairs"] if case == "default" else np.zeros((0, 1), np.int32)
    mw = 0.1 if case in ("default", "walk") else 0.0
    ip = g["indptr"] if case == "walk" else z
    ix = g["indices"] if case == "walk" else z
    b = 1.0 if case == "b1" else 0.8
    mg.optimize_layout(Y, g["head"], g["tail"], eps, eons, eonns, ip, ix, 0, 40, 1.0, 0.0, mw, 0.0, 1.7, b, 1.7382,
                       1.0, 5.0, 0, 1.0, 2.0, 4, 0.25, 0, 0, 0, np.zeros((0, 2), np.float32),
                       np.zeros((0, 2), np.float32), z, 0.9, 0.999, z, mp, z, z, 0.0, 0, np.zeros(0, np.float32),
                       seed, 1, 0, None, None, stream_mode)
    return Y, eons, eonns


purity = C.purity


@pytest.mark.parametrize("stream_mode", [0, 1])
@pytest.mark.parametrize("case", ["default", "b1", "walk"])
def test_layout_against_reference(mg, golden, stream_mode, case):
    g = golden("sgd_small.npz")
    Y, eons, eonns = run_layout(mg, g, stream_mode, case)
    assert np.array_equal(eons, g[f"eons_{case}"]) and np.array_equal(eonns, g[f"eonns_{case}"])
    assert np.isfinite(Y).all()
    # layout quality over 8 seeds against the reference's own 8 runs (same inputs, seeds 1..8): single runs of
    # a 600-point layout spread by a few points of purity, so the means are compared (tolerance 0.03)
    labels = g["labels"]
    p_ref = np.mean([purity(Yr, labels) for Yr in g[f"Yseeds_{case}"]])
    p = np.mean([purity(run_layout(mg, g, stream_mode, case, seed=s)[0], labels) for s in range(1, 9)])
    assert p > p_ref - 0.03, (p, p_ref)


def test_serial_stream_mode_is_deterministic(mg, golden):
    g = golden("sgd_small.npz")
    Y1, _, _ = run_layout(mg, g, 1)
    Y2, _, _ = run_layout(mg, g, 1)
    assert np.array_equal(Y1, Y2)


def test_fixed_points_do_not_move(mg, golden):
    g = golden("sgd_small.npz")
    Y = g["Y0"].copy(); eps = g["eps"]; eons = eps.copy(); eonns = (eps / 5).astype(np.float32)
    z = np.zeros(0, np.int32)
    mg.optimize_layout(Y, g["head"], g["tail"], eps, eons, eonns, z, z, 0, 10, 1.0, 0.5, 0.0, 0.0, 1.7, 0.8, 1.7382,
                       1.0, 5.0, 0, 1.0, 2.0, 4, 0.25, 0, 0, 300, np.zeros((0, 2), np.float32),
                       np.zeros((0, 2), np.float32), z, 0.9, 0.999, z, np.zeros((0, 1), np.int32), z, z, 0.0, 0,
                       np.zeros(0, np.float32), 7, 1, 0)
    assert np.array_equal(Y[:300], g["Y0"][:300])
    assert not np.array_equal(Y[300:], g["Y0"][300:])


def test_argument_errors(mg, golden):
    g = golden("sgd_small.npz")
    Y = g["Y0"].copy(); eps = g["eps"]; eons = eps.copy(); eonns = (eps / 5).astype(np.float32)
    z = np.zeros(0, np.int32)
    bad_head = g["head"].copy(); bad_head[3] = 10 ** 6
    with pytest.raises(RuntimeError, match="edge index out of range"):
        mg.optimize_layout(Y, bad_head, g["tail"], eps, eons, eonns, z, z, 0, 1, 1.0, 1.0, 0.0, 0.0, 1.7, 0.8, 1.7,
                           1.0, 5.0, 0, 1.0, 2.0, 4, 0.25, 0, 0, 0, np.zeros((0, 2), np.float32),
                           np.zeros((0, 2), np.float32), z, 0.9, 0.999, z, np.zeros((0, 1), np.int32), z, z, 0.0, 0,
                           np.zeros(0, np.float32), 7, 1, 0)
    with pytest.raises(RuntimeError, match="loss must be 0"):
        mg.optimize_layout(Y, g["head"], g["tail"], eps, eons, eonns, z, z, 0, 1, 1.0, 1.0, 0.0, 0.0, 1.7, 0.8, 1.7,
                           1.0, 5.0, 3, 1.0, 2.0, 4, 0.25, 0, 0, 0, np.zeros((0, 2), np.float32),
                           np.zeros((0, 2), np.float32), z, 0.9, 0.999, z, np.zeros((0, 1), np.int32), z, z, 0.0, 0,
                           np.zeros(0, np.float32), 7, 1, 0)


SCHEDULE_KEYS = ("epoch_start", "epoch_end", "alpha0", "alpha1", "mid_w0", "mid_w1", "negative_sample_rate", "loss",
                 "mid_rate", "walk_len", "n_fixed", "mid_pairs", "indptr", "indices", "seed", "walk_lens",
                 "jump_indptr", "jump_indices", "mid_jump")


@pytest.mark.parametrize("stream_mode", [1, 0])
@pytest.mark.parametrize("case", C.SCHEDULE_CASES)
def test_option_schedule_bit_exact(mg, golden, stream_mode, case):
    """InfoNCE negatives, jump-graph and per-node-length walks and a 3-d layout: the device's draws of six epochs
    equal the oracle's (the reference's single stream in the serial mode, its per-edge replay in the counter mode)"""
    g = golden("sgd_small.npz")
    Y, e_o, en_o, kw = C.state(g, case)
    _, e_d, en_d, _ = C.state(g, case)
    for epoch in range(6):
        rec_o = O.sgd_schedule(Y.copy(), g["head"], g["tail"], g["eps"], e_o, en_o, epoch,
                               per_edge_stream=(stream_mode == 0), **C.oracle_kw(kw))
        rec_d = mg.layout_schedule(Y.copy(), g["head"], g["tail"], g["eps"], e_d, en_d, epoch,
                                   stream_mode=stream_mode, **{k: kw[k] for k in SCHEDULE_KEYS})
        assert np.array_equal(rec_o[0].astype(bool), rec_d[0].astype(bool))
        for a, b in zip(rec_o[1:], rec_d[1:]):
            assert np.array_equal(a, b)
        assert np.array_equal(e_o, e_d) and np.array_equal(en_o, en_d)


def run_case(mg, g, case, stream_mode, seed=12345):
    Y, eons, eonns, kw = C.state(g, case, seed)
    mg.optimize_layout(Y, g["head"], g["tail"], g["eps"], eons, eonns, n_threads=1, stream_mode=stream_mode, **kw)
    return Y, eons, eonns, kw


@pytest.mark.parametrize("stream_mode", [0, 1])
@pytest.mark.parametrize("case", C.CASES)
def test_option_layout_against_reference(mg, golden, stream_mode, case):
    """each option case on the device: the eons / eonns bookkeeping equals the reference's bit for bit, fixed
    nodes stay put, Adam's per-node step counts equal the oracle's replay of the same draws (counter mode), and the
    layout's 10-NN label purity over seeds 1..8 matches the reference's own 8 runs"""
    g, opts = golden("sgd_small.npz"), golden("sgd_options.npz")
    Y0 = C.state(g, case)[0]
    if stream_mode == 1 and C.state(g, case)[3]["optimizer"] == 1:
        with pytest.raises(RuntimeError, match="supports the sgd optimizer only"):
            run_case(mg, g, case, stream_mode)
        return
    Y, eons, eonns, kw = run_case(mg, g, case, stream_mode)
    _, eons_r, eonns_r = C.expected(g, opts, case)
    assert np.array_equal(eons, eons_r) and np.array_equal(eonns, eonns_r)
    assert np.isfinite(Y).all()
    nf = kw["n_fixed"]
    assert np.array_equal(Y[:nf], Y0[:nf]) and not np.array_equal(Y[nf:], Y0[nf:])
    if kw["optimizer"] == 1:
        Yo, eo, eno, kwo = C.state(g, case)
        O.sgd_serial(Yo, g["head"], g["tail"], g["eps"], eo, eno, per_edge_stream=True, **C.oracle_kw(kwo))
        assert np.array_equal(kw["adam_t"], kwo["adam_t"])
        assert np.isfinite(kw["adam_m"]).all() and (kw["adam_v"] >= 0).all()
    # the reference's own spread over seeds sets the tolerance (InfoNCE and Adam layouts of 40 epochs vary by
    # several points of purity from seed to seed): 8-seed means within max(0.03, 1.5 std)
    p_ref = opts[f"purity_{case}"]
    p = np.mean([purity(run_case(mg, g, case, stream_mode, seed=sd)[0], g["labels"]) for sd in range(1, 9)])
    assert p > p_ref.mean() - max(0.03, 1.5 * p_ref.std()), (p, p_ref.mean())
