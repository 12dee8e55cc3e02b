"""Multi-GPU runs are replicas: every rank deduplicates its own buffers (like the reference's MPI
driver, src/dedup_files_mpi.cpp:54-65), and nothing crosses ranks but a barrier and the
reduction of the measurements below (and an agreement on how the timed steps are grouped).
One buffer does not shard without a digest-partitioned exchange the reference does not have."""
import torch
import torch.distributed as dist


def world():
    return dist.get_world_size() if dist.is_available() and dist.is_initialized() else 1


def reduce_timing(ms, units, device=None):
    """(max over ranks of `ms`, sum over ranks of `units`): the whole-job time is the slowest
    rank's, the whole-job work is everyone's."""
    if world() == 1:
        return float(ms), float(units)
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    u = torch.tensor([float(units)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    return float(t.item()), float(u.item())


def throughput(ms, units, device=None):
    """whole-job units per second over the slowest rank's time"""
    ms_max, total = reduce_timing(ms, units, device)
    return total / (ms_max * 1e-3), ms_max


def agree_min(value, device=None):
    """the smallest `value` over ranks: every rank then takes the same steps in the same groups
    (each group ends in a barrier, so ranks must agree on how many there are)"""
    if world() == 1:
        return int(value)
    t = torch.tensor([int(value)], dtype=torch.int64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MIN)
    return int(t.item())
