"""The N > 1 (replicas) path of bench.py on CPU: two gloo ranks, disjoint
event ranges, device time reduced as the max over ranks, and the whole
harness (process group, event partition, timing reduction, the one JSON line
of rank 0) run end to end with the GPU replica replaced by a stub.  The
replicas are not measured on GPUs here: this run has one GPU."""
import json
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


def _stub_replica(args, rank, world, local, events):
    """Stands in for bench.run_ours: records which events the rank got and
    reduces a rank-dependent 'device time' the way run_ours does."""
    import bench
    from tracklooper_b200 import gen

    firsts = [gen.event_seed(args.config, bench.rank_first_event(rank, args.batch) + i) for i in range(len(events))]
    hits = [int(e.n_hits) for e in events]
    ms = bench.reduce_max(100.0 * (rank + 1) * args.steps, world)
    return {"value": args.batch * world * args.steps / (ms * 1e-3), "ms_per_step": ms / args.steps,
            "stub": {"rank": rank, "seeds": firsts, "hits": hits}}


def _harness_rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import contextlib
    import io

    import bench

    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        bench.main(["--gpus", str(world), "--batch", "2", "--config", "1", "--steps", "3", "--warmup", "3"],
                   runner=_stub_replica, backend="gloo")
    out.put((rank, buf.getvalue()))


def test_harness_end_to_end_two_gloo_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_harness_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=240) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs)
    assert res[1].strip() == ""  # only rank 0 prints
    lines = [ln for ln in res[0].splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["n_gpus"] == 2 and line["scaling"] == "weak"
    assert line["config"]["parallelism"] == "replicas x2"
    # the value counts both ranks' events over the slower rank's time
    assert abs(line["value"] - 2 * 2 * 3 / (200.0 * 3 * 1e-3)) < 1e-9
    assert line["stub"]["rank"] == 0


def test_launcher_spawns_one_process_per_gpu():
    import bench

    cmd = bench.launcher_command(["--gpus", "4", "--steps", "2"], 4, 29555)
    assert cmd[1:3] == ["-m", "torch.distributed.run"]
    assert "--nproc-per-node=4" in cmd and "127.0.0.1" in cmd and "--master-port=29555" in cmd
    assert cmd[-4:] == ["--gpus", "4", "--steps", "2"] and cmd[-5].endswith("bench.py")
