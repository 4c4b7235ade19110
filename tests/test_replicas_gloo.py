"""Multi-process (world size 2, gloo, CPU) checks of the replica plumbing that
bench.py uses for N > 1 GPUs: slices cover the batch exactly once, per-rank
seeds differ, the elapsed-time reduction returns the slowest rank, and the
barrier releases every rank."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from sunny_gen_eigensolver_b200.replicas import partition, rank_seed


def test_partition_covers_exactly_once():
    for total in (0, 1, 7, 65536, 1_000_003):
        for world in (1, 2, 3, 8):
            got = [partition(total, world, r) for r in range(world)]
            assert got[0][0] == 0 and got[-1][1] == total
            assert all(got[i][1] == got[i + 1][0] for i in range(world - 1))
            sizes = [b - a for a, b in got]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        partition(10, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    from sunny_gen_eigensolver_b200 import replicas
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        replicas.barrier()
        t = replicas.max_over_ranks(1.5 + rank)          # rank 1 is the slow one
        start, stop = replicas.partition(10, world, rank)
        q.put((rank, t, start, stop, replicas.rank_seed(7, rank)))
        replicas.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_reduction_and_barrier():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [2.5, 2.5]
    assert (out[0][2], out[0][3], out[1][2], out[1][3]) == (0, 5, 5, 10)
    assert out[0][4] != out[1][4] == rank_seed(7, 1)
