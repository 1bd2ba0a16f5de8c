"""The N > 1 (replicas) path of bench.py on CPU: two gloo ranks, disjoint
event ranges, device time reduced as the max over ranks."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime

    import torch.distributed as tdist

    import bench

    tdist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        first = bench.rank_first_event(rank, 64)
        ms = bench.reduce_max(10.0 + 5.0 * rank, world)
        out.put((rank, first, ms))
    finally:
        tdist.destroy_process_group()


def test_two_ranks_take_disjoint_events_and_max_time():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(q.get(timeout=5) for _ in range(2))
    assert [r[1] for r in res] == [0, 64]
    assert all(r[2] == 15.0 for r in res)


def test_single_rank_reduce_is_identity():
    import bench

    assert bench.reduce_max(3.5, 1) == 3.5
