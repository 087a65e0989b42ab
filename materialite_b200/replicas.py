"""Multi-GPU serving by replicas: one process per GPU, each with its own RVE server.

One RVE solve does not shard: its 3-D FFT needs global transposes. Independent requests
do shard, so N GPUs serve N disjoint parts of the request stream with no collective on
the solve path. The only collectives are on the host side: a barrier around timed
regions and max/sum reductions of scalars. They run over NCCL on GPUs and over gloo in
the CPU tests.
"""

import datetime
import os

import numpy as np


def rank_info():
    """(world, rank, local_rank) from the torchrun environment (1, 0, 0 without it)."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend="nccl", timeout_s=600):
    """Join the process group when WORLD_SIZE > 1. Returns (world, rank, local_rank).
    With NCCL each rank binds the GPU of its local rank."""
    world, rank, local = rank_info()
    if world > 1:
        import torch
        import torch.distributed as dist
        kw = {}
        if backend == "nccl":
            torch.cuda.set_device(local)
            kw["device_id"] = torch.device("cuda", local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
    return world, rank, local


def _device(local):
    import torch.distributed as dist
    return f"cuda:{local}" if dist.get_backend() == "nccl" else "cpu"


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def _reduce(x, world, local, op):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device(local))
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(x, world, local):
    import torch.distributed as dist
    return x if world == 1 else _reduce(x, world, local, dist.ReduceOp.MAX)


def sum_over_ranks(x, world, local):
    import torch.distributed as dist
    return x if world == 1 else _reduce(x, world, local, dist.ReduceOp.SUM)


def request_cost(r):
    """Relative device cost of a request: voxels x steps; crystal plasticity about 8x
    elastic per step (measured Newton x Krylov iteration counts of the serving mix)."""
    w = 8.0 if str(getattr(r, "kind", "")).startswith("evp") else 1.0
    return float(np.prod(r.dims)) * r.steps * w


def partition(requests, world, rank):
    """This rank's share of a request stream: longest-processing-time-first assignment by
    request_cost. Ties break by submission order, so every rank computes the same
    disjoint assignment with no communication."""
    order = sorted(range(len(requests)), key=lambda i: (-request_cost(requests[i]), i))
    load = [0.0] * world
    owner = [0] * len(requests)
    for i in order:
        k = min(range(world), key=lambda j: (load[j], j))
        owner[i] = k
        load[k] += request_cost(requests[i])
    return [r for i, r in enumerate(requests) if owner[i] == rank]


def destroy(world):
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
