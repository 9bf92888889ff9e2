"""Replica layer for several GPUs of one node: one process per GPU, each
solving its own right-hand-side blocks (or its own systems) with no data-path
collective; the only communication is timing and bookkeeping over
torch.distributed (NCCL on GPUs, gloo on CPU).

XAMG's solve phase distributes one system's rows over MPI ranks with a halo
exchange per SpMV (src/comm/matvec_comm.h:203-312); independent right-hand
sides need none of that, which is how the multi-RHS workloads scale here.
"""
import os


def dist_env():
    """(world size, rank, local rank) from the torchrun environment."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def rhs_blocks(total_blocks, world, rank):
    """Indices of the right-hand-side blocks this rank solves: a contiguous
    share, the first total_blocks % world ranks taking one more."""
    if total_blocks < 0 or world < 1 or not 0 <= rank < world:
        raise ValueError("bad block partition arguments")
    base, extra = divmod(total_blocks, world)
    start = rank * base + min(rank, extra)
    return list(range(start, start + base + (1 if rank < extra else 0)))


def assign_systems(work, world):
    """Rank of each independent system: largest work first, each to the
    rank with the least work so far (ties to the lower rank). Every rank
    computes the same assignment from the same work list, so no message is
    needed."""
    if world < 1:
        raise ValueError("world must be at least 1")
    load = [0.0] * world
    owner = [0] * len(work)
    for i in sorted(range(len(work)), key=lambda j: (-work[j], j)):
        r = min(range(world), key=lambda q: (load[q], q))
        owner[i] = r
        load[r] += work[i]
    return owner


def _device(dist):
    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def max_over_ranks(value):
    """Maximum of a per-rank float over all ranks (identity without a
    process group)."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=_device(dist))
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value):
    """Sum of a per-rank count over all ranks."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=_device(dist))
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()
