"""Multi-GPU plumbing for bundle adjustment: independent windows, one per rank.

The BA path has no exchange step.  HI-SLAM2 runs one optimisation window per
process (``hislam2/factor_graph.py`` calls ``droid_backends.ba`` on its own
keyframes and edges), so on N GPUs each rank -- one process per GPU -- solves its
own window with its own workspace, and the ranks are replicas.  The only
collectives are for timing: a barrier on each side of the timed region and a MAX
reduce of every rank's device-timed duration.  Whole-job throughput is the units
all ranks processed divided by the slowest rank's time.
"""

import datetime
import os

import torch


def env_ranks():
    """(world, rank, local_rank) from the launcher's environment (torchrun sets them)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    return world, rank, local


def init(world, local, backend="nccl", timeout_s=180):
    """Joins the process group of `world` ranks (no-op for one rank).  With NCCL the
    rank binds GPU `local` first; the short timeout turns a missing rank into an error."""
    if world <= 1:
        return
    timeout = datetime.timedelta(seconds=timeout_s)
    if backend == "nccl":
        torch.cuda.set_device(local)
        torch.distributed.init_process_group("nccl", timeout=timeout, device_id=torch.device("cuda", local))
    else:
        torch.distributed.init_process_group(backend, timeout=timeout)


def finalize(world):
    if world > 1 and torch.distributed.is_initialized():
        torch.distributed.destroy_process_group()


def barrier(world):
    if world > 1:
        torch.distributed.barrier()


def max_over_ranks(x, world, device=None):
    """The maximum of the float `x` over all ranks (every rank gets it)."""
    if world <= 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def throughput(units_per_rank, max_ms, world):
    """Whole-job rate: the units every rank processed over the slowest rank's time."""
    if max_ms <= 0:
        raise ValueError("max_ms must be positive")
    return units_per_rank * world / (max_ms / 1e3)


def shard(num_windows, world, rank):
    """The windows rank `rank` solves when `num_windows` are spread over `world` ranks:
    a contiguous block, sizes differing by at most one, covering every window once."""
    if not 0 <= rank < world:
        raise ValueError("rank %d outside world of %d" % (rank, world))
    base, extra = divmod(num_windows, world)
    lo = rank * base + min(rank, extra)
    return range(lo, lo + base + (1 if rank < extra else 0))


def window_seed(rank, base=0):
    """Seed of the synthetic window a rank solves (distinct per rank)."""
    return base + rank
