"""The multi-GPU plumbing on the host (replicas only: no collective on the data path): two gloo ranks on the CPU take
the max of their timings the way bench.py's ranks do over NCCL, and a batch of independent geometries is dealt so that
every molecule lands on exactly one rank. CPU only."""
import os
import socket
import sys

import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "atomic-sandbox_b200"))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import torch.distributed as dist
    import ks_replicas as rp
    assert rp.rank_info() == (rank, world, rank)
    rp.init("gloo", timeout_s=60)
    try:
        local = [1.5 + rank, 10.0 - rank, -3.0 * rank]
        got = rp.max_over_ranks(local, "cpu")
        jobs = list(range(13))
        mine = rp.shard(jobs, rank, world)
        sizes = rp.max_over_ranks([len(mine)], "cpu")
        dist.barrier()
        out.put((rank, got, mine, sizes))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_max_and_shard():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got, mine, sizes in res:
        assert got == [2.5, 10.0, 0.0], "the element-wise max over both ranks on every rank"
        assert sizes == [7.0]
    assert sorted(res[0][2] + res[1][2]) == list(range(13)) and not set(res[0][2]) & set(res[1][2])


def test_one_rank_needs_no_process_group():
    import ks_replicas as rp
    assert rp.max_over_ranks([1.0, 2.0], "cpu") == [1.0, 2.0]
    assert rp.shard(range(5), 0, 1) == [0, 1, 2, 3, 4]
