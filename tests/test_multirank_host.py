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
