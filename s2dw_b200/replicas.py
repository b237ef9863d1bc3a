"""Independent replicas across ranks (one process per GPU).

The transform has no cross-GPU exchange: every rank transforms its own maps.
The only collectives are for timing (barrier, max of elapsed time over ranks)
and for checking that every rank finished; they run over NCCL on GPUs or gloo
on CPU with the same code.
"""
import datetime
import os


def rank_info():
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init_group(backend=None, timeout_s=120):
    """Joins the process group when WORLD_SIZE > 1; returns (world, rank, local)."""
    world, rank, local = rank_info()
    if world > 1:
        import torch
        import torch.distributed as dist

        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return world, rank, local


def _device():
    import torch
    import torch.distributed as dist

    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x, world):
    """Maximum of a float over all ranks (the whole job takes as long as its
    slowest rank)."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x, world):
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def finish(world):
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
