"""Replicas on several processes (bench.py --gpus N under torchrun): every rank times its own
replica and the job reports the slowest rank's time, aggregated over the ranks. The host side of
that path runs here on CPU ranks with the gloo backend (world size 2), as the GPU ranks run it
with NCCL: bench.max_over_ranks and the aggregate throughput."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        elapsed = 1.0 + rank  # rank r took 1 + r seconds
        t = bench.max_over_ranks(elapsed, "cpu")
        dist.barrier()
        out.put((rank, t, world * 100.0 / t))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for rank, t, value in got:
        assert t == 2.0          # the slowest rank's time on every rank
        assert value == 100.0    # 2 replicas x 100 units / 2 s


def test_max_over_ranks_single_process():
    import bench
    assert bench.max_over_ranks(3.5, "cpu") == 3.5
