"""Multi-GPU replicas: one process per GPU, each holding its own copy of the
gauge configuration and solving its own share of independent right-hand
sides or requests.

The solver path needs no data exchange between GPUs (every solve is
independent), so there is no collective on the data path.  The only
collectives are host-side bookkeeping: the maximum over ranks of a device
time (a whole-job rate is the work of all ranks over the slowest rank's
time), and the gathering of per-request results to rank 0.  They run on
whatever process group is initialised (NCCL on GPUs, gloo on CPU).
"""
from __future__ import annotations

import os


def dist_env():
    """(world_size, rank, local_rank) from the torchrun environment (1, 0, 0 without it)."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def share(items, rank: int, world: int):
    """This rank's share of a sequence of independent work items (round robin)."""
    return list(items)[rank::world]


def rank_columns(rank: int, steps: int, ncol: int = 12):
    """Spin-colour columns a rank solves in `steps` solves: every rank cycles
    through the 12 columns from its own offset, so each rank does the same
    amount of work as a single GPU would."""
    return [(rank * steps + k) % ncol for k in range(steps)]


def _reduce_device(group):
    import torch
    import torch.distributed as dist
    backend = dist.get_backend(group)
    return torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")


def max_over_ranks(x: float, group=None) -> float:
    """Maximum of a per-rank scalar over all ranks (identity without a process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_reduce_device(group))
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def whole_job_rate(units_per_rank: float, ms_max: float, world: int) -> float:
    """Units per second of the whole job: all ranks' units over the slowest rank's time."""
    return world * units_per_rank / (ms_max * 1e-3)


def gather_to_root(obj, group=None):
    """List of every rank's `obj` on rank 0 (None elsewhere); [obj] without a process group."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return [obj]
    world = dist.get_world_size(group)
    out = [None] * world if dist.get_rank(group) == 0 else None
    dist.gather_object(obj, out, dst=0, group=group)
    return out


def serve_share(schedule, rank: int, world: int):
    """This rank's requests of a (time, request) schedule: request i goes to rank i % world,
    arrival times unchanged (each rank runs its own server on its own GPU)."""
    return [item for i, item in enumerate(schedule) if i % world == rank]
