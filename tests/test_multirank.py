"""Multi-process host logic of bench.py on CPU (gloo, world size 2): each rank
takes its own disjoint block of consecutive primes (no data-path collective),
the step time is the maximum over ranks and the profiles counted are the sum
of every rank's own block."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    ps = bench.workload(rank)
    t = bench.max_over_ranks([10.0 * (rank + 1), 1.0], dist, "cpu")
    total = bench.sum_over_ranks(100.0 + rank, dist, "cpu")
    q.put((rank, ps[0], ps[-1], len(ps), t, total))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_disjoint_blocks_and_max_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, a0, b0, n0, t0, s0), (r1, a1, b1, n1, t1, s1) = res
    assert n0 == n1 == 4096
    assert b0 == 4294967291 and b1 < a0          # rank 1's block lies below rank 0's
    assert t0 == t1 == [20.0, 1.0]               # maximum over ranks on every rank
    assert s0 == s1 == 201.0                     # per-rank counts summed on every rank
