"""The bench's multi-GPU host logic on CPU: N replicas (one circuit per
rank, no data-path collective), step time = max over ranks. Two gloo ranks
on 127.0.0.1 stand in for the GPUs."""

import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # Each replica measured a different step time; all must report the max.
        value = bench.max_over_ranks(0.25 + 0.5 * rank, dist, device="cpu")
        dist.barrier()
        out.put((rank, value, bench.max_over_ranks(3.0, None)))
    finally:
        dist.destroy_process_group()


def test_replicas_report_the_max_over_ranks():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(out.get(timeout=10) for _ in range(2))
    assert [g[1] for g in got] == [0.75, 0.75]
    assert all(g[2] == 3.0 for g in got)
