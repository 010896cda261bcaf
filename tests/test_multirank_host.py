"""The multi-rank path of bench.py on the host: two gloo ranks on CPU (127.0.0.1). A single layout runs on one GPU
(replicas only, no data-path collective); across ranks the job's time is the slowest rank's, every rank takes the
same collective steps, and the whole job's seconds per layout divides it by the number of replicas."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank, world, port, out):
    import datetime
    import sys
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench as B
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        step_ms = 100.0 + 50.0 * rank              # the ranks' own step times differ
        ms = B.max_over_ranks(step_ms, dist)
        e2e = B.max_over_ranks(120.0 + 30.0 * (world - 1 - rank), dist)
        dist.barrier()
        out[rank] = (ms, e2e, B.seconds_per_layout(ms, world))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks_take_the_slowest_rank():
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    port = free_port()
    procs = [ctx.Process(target=rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    assert out[0] == out[1] == (150.0, 150.0, 0.075)


def test_single_rank_needs_no_collective():
    import bench as B
    assert B.max_over_ranks(42.5) == 42.5
    assert B.seconds_per_layout(482.0, 1) == 0.482


def small_layout(i):
    """item i of the replica test: a seeded SGD layout of 200-700 points (the oracle's restatement of the
    reference's single-stream SGD, deterministic, so the result does not depend on which rank runs it)"""
    import numpy as np
    from oracle import oracle as O
    rng = np.random.default_rng(100 + i)
    n = int(rng.integers(200, 700))
    head = np.repeat(np.arange(n, dtype=np.int32), 6)
    tail = ((head + rng.integers(1, n, head.size)) % n).astype(np.int32)
    eps = rng.uniform(1.0, 3.0, head.size).astype(np.float32)
    Y = rng.uniform(-5, 5, (n, 2)).astype(np.float32)
    O.sgd_serial(Y, head, tail, eps, eps.copy(), (eps / 5).astype(np.float32), a=1.6, b=0.9, seed=i, epoch_start=0,
                 epoch_end=15, alpha0=1.0, alpha1=0.1)
    return n, Y


def replica_main(rank, world, port, out):
    import datetime
    import sys
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (root, os.path.join(root, "lib-magnet_b200")):
        sys.path.insert(0, p)
    from magnet_b200 import replicas as Rp
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        sizes = [Rp.layout_bytes(200 + 50 * i, 3000 * (i + 1)) for i in range(7)]
        free = [10 ** 9 + rank * 1000]           # the ranks' own free memory differs
        all_free = [None] * world
        dist.all_gather_object(all_free, free[0])
        owner = Rp.place(sizes, all_free)
        mine = Rp.share(owner, rank)
        res = Rp.gather_results([(i, small_layout(i)) for i in mine], dist)
        out[rank] = (owner, mine, [(n, Y.tobytes()) for n, Y in res])
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_two_gloo_ranks_split_layouts_and_merge():
    """each rank places the same items by free memory, runs only its share, and the merged results equal a
    one-rank run of all items, bit for bit"""
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    port = free_port()
    procs = [ctx.Process(target=replica_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(150)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    (own0, mine0, res0), (own1, mine1, res1) = out[0], out[1]
    assert own0 == own1 and sorted(mine0 + mine1) == list(range(7)) and mine0 and mine1
    solo = [small_layout(i) for i in range(7)]
    assert res0 == res1 == [(n, Y.tobytes()) for n, Y in solo]


def test_placement_by_free_memory():
    from magnet_b200 import replicas as Rp
    owner = Rp.place([50, 40, 30, 20, 10], [60, 100])
    assert owner == [1, 0, 1, 0, 1]                # decreasing size, each to the most free memory left
    assert Rp.share(owner, 0) == [1, 3]
    with pytest.raises(ValueError):
        Rp.place([200], [100, 150])
    assert Rp.gather_results([(2, "c"), (0, "a"), (1, "b")]) == ["a", "b", "c"]
