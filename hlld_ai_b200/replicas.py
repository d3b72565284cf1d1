"""Host plumbing of replica runs: one process per GPU under torchrun.

The 2D step has no domain decomposition (the reference runs one process
with intra-op threads), and batched tubes are independent units, so a run
on N GPUs is N replicas: every rank advances its own rotor or its own
seeded tube batch, and the only collectives are a barrier and the
reductions that turn per-rank timings into one whole-job number -- the
slowest rank's time (MAX) and, for tubes, the total work (SUM).

The collectives run on whatever backend the process group has: NCCL on
the GPUs, gloo on CPU for the host-side tests.  Every rank takes the same
collective steps in the same order.
"""
from __future__ import annotations

import datetime
import os
from dataclasses import dataclass

import torch
import torch.distributed as dist


@dataclass(frozen=True)
class Replica:
    world: int  # number of ranks
    rank: int  # this rank
    local: int  # this rank's device index on its node
    device: torch.device  # where the reduction tensors live


def from_env(device_type: str = "cuda") -> Replica:
    """RANK / LOCAL_RANK / WORLD_SIZE as torchrun sets them (1 rank without)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dev = torch.device("cuda", local) if device_type == "cuda" else torch.device("cpu")
    return Replica(world, rank, local, dev)


def init(r: Replica, timeout_s: float = 300.0) -> None:
    """Join the process group when there is more than one rank: NCCL for CUDA
    devices, gloo otherwise.  A short timeout makes ranks that wait for a
    missing peer end with an error instead of hanging."""
    if r.world <= 1:
        return
    timeout = datetime.timedelta(seconds=timeout_s)
    if r.device.type == "cuda":
        dist.init_process_group("nccl", device_id=r.device, timeout=timeout)
    else:
        dist.init_process_group("gloo", timeout=timeout)


def barrier(r: Replica) -> None:
    if r.world > 1:
        dist.barrier()


def max_over_ranks(r: Replica, *values: float) -> list[float]:
    """Element-wise maximum over ranks (the slowest rank's time)."""
    if r.world <= 1:
        return [float(v) for v in values]
    t = torch.tensor(values, dtype=torch.float64, device=r.device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


def sum_over_ranks(r: Replica, *values: float) -> list[float]:
    """Element-wise sum over ranks (the whole job's work)."""
    if r.world <= 1:
        return [float(v) for v in values]
    t = torch.tensor(values, dtype=torch.float64, device=r.device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return [float(x) for x in t.tolist()]


def job_rate(r: Replica, units_per_rank: float, ms_local: float) -> tuple[float, float]:
    """Whole-job throughput of equal replicas (weak scaling): all ranks' units
    over the slowest rank's time.  Returns (units per second, that time in ms)."""
    (ms,) = max_over_ranks(r, ms_local)
    return r.world * units_per_rank / (ms * 1e-3), ms


def replica_seed(base: int, r: Replica) -> int:
    """Each rank's own seed for independent work units (tube batches)."""
    return base + r.rank


def finish(r: Replica) -> None:
    """Last barrier and leave the process group."""
    if r.world > 1:
        dist.barrier()
        dist.destroy_process_group()
