"""Replica runs on several GPUs of one node.

One process per GPU (launched by torchrun), each advancing its own
independent mesh: the Lagrange + remap step has no exchange between separate
meshes, so there is no data collective.  The only communication is a barrier
around the timed region and the maximum of the per-rank times, so that the
whole-job throughput is all ranks' cell-cycles over the slowest rank's time.
"""
from __future__ import annotations

import datetime
import os

import torch
import torch.distributed as dist


def ranks():
    """(world size, rank, local rank) from the launcher's environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def partition(weights, world: int, rank: int) -> list[int]:
    """Indices of the instances that rank runs, split by cell count: the
    heaviest first, each to the least-loaded rank (ties to the lower rank),
    returned in increasing order.  Every rank computes the same split with no
    exchange; with 64 instances of 32^3..96^3 cells the heaviest of 8 ranks
    carries 1.003x the mean (round-robin: 1.39x)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    load = [0.0] * world
    owner = [0] * len(weights)
    for i in sorted(range(len(weights)), key=lambda i: (-float(weights[i]), i)):
        r = min(range(world), key=lambda r: (load[r], r))
        load[r] += float(weights[i])
        owner[i] = r
    return [i for i in range(len(weights)) if owner[i] == rank]


def init(backend: str, device=None, timeout_s: float = 300.0) -> None:
    """Process group over MASTER_ADDR/MASTER_PORT; a short timeout makes a rank
    that never arrives end the others' collectives with an error."""
    kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
    if device is not None and backend == "nccl":
        kw["device_id"] = device
    dist.init_process_group(backend, **kw)


def active() -> bool:
    return dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1


def barrier() -> None:
    if active():
        dist.barrier()


def max_over_ranks(x: float, device="cpu") -> float:
    if not active():
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, device="cpu") -> float:
    if not active():
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def aggregate(units_local: float, steps: int, ms_local: float, device="cpu"):
    """(slowest rank's ms, whole-job units per second): the units all ranks
    processed (replicas may differ in size) over the slowest rank's time."""
    ms = max_over_ranks(ms_local, device)
    units = sum_over_ranks(units_local, device)
    return ms, units * steps / (ms / 1e3)


def finish() -> None:
    if dist.is_available() and dist.is_initialized():
        dist.destroy_process_group()
