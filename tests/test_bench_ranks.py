"""bench.py's multi-process logic on CPU: with world_size 2 over gloo, every
rank gets the slowest rank's time from RankSync.max, the barrier returns on
both, and the process group closes cleanly (the same calls the NCCL ranks of
`torchrun --nproc-per-node N bench.py --gpus N` make)."""
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, q):
    import os
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import bench
    sync = bench.RankSync(world, backend="gloo", timeout_s=60)
    sync.barrier()
    slowest = sync.max(1.5 + rank)
    sync.barrier()
    sync.close()
    q.put((rank, slowest))


def test_two_gloo_ranks_agree_on_the_slowest():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        got = sorted(q.get(timeout=120) for _ in procs)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert got == [(0, 2.5), (1, 2.5)]
    assert all(p.exitcode == 0 for p in procs)


def test_single_rank_is_a_no_op():
    import bench
    sync = bench.RankSync(1, backend="gloo")
    sync.barrier()
    assert sync.max(3.25) == 3.25
    sync.close()
