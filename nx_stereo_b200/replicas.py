"""Independent replicas across ranks: the multi-GPU form of this path.

Pairs and camera streams are independent and every SGM path crosses the
whole image, so a pair is never split across GPUs and no data moves between
them: each rank (one process per GPU) matches its own pairs. The only
collective is the timing reduction: the job takes as long as its slowest
rank, and its throughput is every rank's units over that time.
"""
import datetime
import os


def ranks():
    """(rank, world_size, local_rank) from the launcher's environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend, rank=None, world_size=None, device=None, timeout_s=120, init_method=None):
    """Joins the process group (nccl for GPUs, gloo for host-only ranks)."""
    import torch.distributed as dist

    kwargs = {"timeout": datetime.timedelta(seconds=timeout_s)}
    if init_method:
        kwargs.update(init_method=init_method, rank=rank, world_size=world_size)
    if device is not None:
        kwargs["device_id"] = device
    dist.init_process_group(backend, **kwargs)


def max_over_ranks(value, device="cpu"):
    """The largest `value` over all ranks (the value itself with one rank)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def agree(flag, device="cpu"):
    """Rank 0's `flag` on every rank (the flag itself with one rank), so that
    every rank takes the same number of rounds of a loop with collectives."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return bool(flag)
    t = torch.tensor([1 if flag else 0], dtype=torch.int32, device=device)
    dist.broadcast(t, src=0)
    return bool(t.item())


def barrier():
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized():
        dist.barrier()


def whole_job_rate(units_per_rank, world_size, slowest_seconds):
    """Units every rank processed over the slowest rank's time."""
    return units_per_rank * world_size / slowest_seconds


def seed(rank, index):
    """A distinct input seed for each rank and pair."""
    return 1_000_003 * (rank + 1) + index
