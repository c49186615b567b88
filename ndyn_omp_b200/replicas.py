"""One process per GPU, replicas only.

The timestep path has no exchange between systems: N ranks each step their
own systems and nothing crosses ranks but timing (the slowest rank's time)
and totals.  torch.distributed carries those two reductions: NCCL between
GPU ranks, gloo on CPU (tests).  A list of independent items (replicas,
requests) is dealt round-robin so every rank's share differs by at most one.
"""
import datetime
import os


def init(timeout_s=120):
    """(world, rank, local_rank) from the launcher's environment; joins the
    process group when world > 1 (NCCL when CUDA is present, else gloo)."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import torch
        import torch.distributed as dist
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=timeout_s),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=timeout_s))
    return ws, rank, local


def _tensor(x):
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    return torch.tensor([float(x)], dtype=torch.float64, device=dev)


def reduce_max(x, ws):
    """max of x over ranks (the job's time is its slowest rank's)"""
    if ws == 1:
        return float(x)
    import torch.distributed as dist
    t = _tensor(x)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(x, ws):
    if ws == 1:
        return float(x)
    import torch.distributed as dist
    t = _tensor(x)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def shard(items, rank, ws):
    """this rank's items, dealt round-robin"""
    return list(items)[rank::ws]


def finish(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
