"""One process per GPU: rank bookkeeping and the host-side steps that cross ranks.

The raster workloads of this engine shard without any exchange on the data
path: every rank evaluates its own rasters (weak scaling), serving runs one
server per GPU over its own DEM replica, and the radial / spreading scans are
per request. What crosses ranks is only timing and synchronisation: a barrier
around the timed region and the slowest rank's time (an all-reduce MAX over
one number), from which the whole job's throughput is computed. This module
holds those steps so that they run, and are tested, on any torch.distributed
backend: NCCL on GPUs, gloo on CPU.
"""
import datetime
import os


def rank_info(env=None):
    """(rank, local_rank, world_size) from the launcher's environment."""
    env = os.environ if env is None else env
    return int(env.get("RANK", "0")), int(env.get("LOCAL_RANK", "0")), int(env.get("WORLD_SIZE", "1"))


def init(backend, world, timeout_s=300):
    """Joins the process group when world > 1; returns torch.distributed or None."""
    if world <= 1:
        return None
    import torch.distributed as dist
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def barrier(dist):
    if dist is not None:
        dist.barrier()


def max_over_ranks(value, dist, device=None):
    """The largest `value` over all ranks (every rank receives it)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(units_per_rank, world, slowest_ms):
    """Whole-job units per second when every rank processes `units_per_rank`
    and the slowest rank takes `slowest_ms`."""
    return units_per_rank * world / (slowest_ms * 1e-3)


def shard(costs, rank, world):
    """Indices of the items this rank takes: items sorted by decreasing cost,
    each given to the rank with the least total so far (ties to the lowest
    rank). Every rank computes the same assignment from the same costs."""
    loads = [0.0] * world
    owner = [0] * len(costs)
    for i in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        r = min(range(world), key=lambda q: (loads[q], q))
        owner[i] = r
        loads[r] += costs[i]
    return [i for i in range(len(costs)) if owner[i] == rank]


def finish(dist):
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
