"""The multi-GPU path of bench.py is replicas: each rank analyses its own segments and the ranks
meet only to take the max of their times.  Two gloo ranks on the CPU check that logic."""

import datetime
import os
import socket

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    out = bench.combine_ranks([1.0 + rank, 10.0 - 3 * rank], dist)
    env = bench.dist_env()
    q.put((rank, out, bench.segment_seed(rank), env))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_replicas_take_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    got.sort()
    for rank, out, seed, env in got:
        assert out == [2.0, 10.0]            # max over ranks, identical on both
        assert env == (rank, 2, rank)
    assert got[0][2] != got[1][2]            # each replica has its own segments


def test_single_process_needs_no_group():
    import sys
    sys.path.insert(0, ROOT)
    import bench
    assert bench.combine_ranks([3.0, 4.0], None) == [3.0, 4.0]
