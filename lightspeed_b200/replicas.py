"""Replica runs over torch.distributed, one process per GPU.

A J/K build is not sharded across GPUs here: each rank builds J and K for
its own copy of the workload (weak scaling), so the data path has no
collective. The only collectives are the barriers around a timed region and
one all-reduce that takes the maximum of each timing over the ranks; every
rank issues them in the same order. Whole-job throughput is then the units
all ranks processed divided by that maximum time.
"""
import os
from datetime import timedelta


def dist_info():
    """(rank, world size, local rank) from the launcher's environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def _dist():
    import torch.distributed as dist
    return dist


def active():
    """True when a process group spans more than one rank."""
    dist = _dist()
    return dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1


def init(backend="nccl", timeout_s=600):
    """Join the process group when the launcher started more than one rank
    (MASTER_ADDR/MASTER_PORT from the environment); a short timeout turns a
    rank that never arrives into an error on the others."""
    _, world, _ = dist_info()
    if world > 1:
        _dist().init_process_group(backend, timeout=timedelta(seconds=timeout_s))


def barrier():
    if active():
        _dist().barrier()


def max_over_ranks(values, device="cpu"):
    """The elementwise maximum of a list of floats over all ranks (one
    all-reduce); the list itself on a single rank."""
    values = [float(v) for v in values]
    if not active():
        return values
    import torch
    t = torch.tensor(values, dtype=torch.float64, device=device)
    _dist().all_reduce(t, op=_dist().ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def whole_job_rate(units_per_rank, world, seconds):
    """Units per second of the whole job: every rank processed units_per_rank
    in at most `seconds` (the max over ranks)."""
    return world * units_per_rank / seconds


def finish():
    if _dist().is_available() and _dist().is_initialized():
        _dist().destroy_process_group()
