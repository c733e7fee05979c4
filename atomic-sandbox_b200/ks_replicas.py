"""Replica plumbing for runs on several GPUs of one node: one process per GPU (torchrun), no collective on the data
path. The SCF of one molecule does not shard (the reference solves on one GPU), so N GPUs run N independent solves,
or deal a batch of independent geometries round-robin; the only collectives are the barrier around a timed region
and the max over ranks of its time (a device-side reduction over NCCL on GPUs, gloo on the host in the tests)."""
import datetime
import os


def rank_info():
    """(rank, world size, local rank) from the torchrun environment; (0, 1, 0) when run alone."""
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def init(backend, device=None, timeout_s=300):
    """Joins the process group (127.0.0.1 rendezvous from the environment) with a bounded timeout, so that ranks which
    wait for one another end with an error instead of hanging."""
    import torch.distributed as dist
    kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
    if device is not None:
        kw["device_id"] = device
    dist.init_process_group(backend, **kw)


def max_over_ranks(values, device):
    """Element-wise max of a list of floats over all ranks (each rank passes its own); the values unchanged when the
    process group is not initialised (one rank)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [float(v) for v in values]
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def shard(items, rank, world):
    """This rank's share of a batch of independent geometries: round-robin, every item on exactly one rank."""
    return list(items)[rank::world]
