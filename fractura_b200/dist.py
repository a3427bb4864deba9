"""Multi-process plumbing for one-process-per-GPU runs (torch.distributed).

The escape-time path has no data-path exchange when every rank renders its own
frames, so ranks only meet to line up their timed regions and to agree on the
slowest rank's time.  The helpers work on any backend: NCCL ranks reduce on
their GPU, gloo ranks on the CPU.
"""
import os

import torch
import torch.distributed as dist


def env():
    """(rank, world_size, local_rank) from the launcher's environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def active():
    return dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1


def _device():
    return torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" \
        else torch.device("cpu")


def barrier():
    if active():
        dist.barrier()


def max_over_ranks(x):
    """The largest value of x over all ranks (x itself on one rank)."""
    if not active():
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x):
    if not active():
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def whole_job_rate(units_per_rank, steps, world, slowest_ms):
    """Aggregate throughput of a weak-scaling run: every rank processes
    units_per_rank per step; the job takes as long as its slowest rank."""
    if slowest_ms <= 0.0:
        raise ValueError("slowest_ms must be positive")
    return units_per_rank * steps * world / (slowest_ms * 1e-3)
