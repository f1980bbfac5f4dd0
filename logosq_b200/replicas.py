"""One process per GPU: rank plumbing for the benchmark and the batched engine.

The dense single-state path does not shard: N GPUs run N independent replicas
and the job's throughput is N x the units of one replica over the slowest
rank's time.  The batched VQE engine does partition: its instances are
independent, so each rank takes a cost-balanced share of them and no data
crosses between ranks during a step (the only collective is the timing
reduction).  The reference has no multi-process layer (its parallelism is
rayon threads inside one process, e.g. src/states/mod.rs:244-258, 350-365).
"""
from __future__ import annotations

import datetime
import os


def dist_info():
    """(world size, rank, local rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: int = 300) -> None:
    import torch.distributed as dist
    if not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))


def _device():
    import torch
    import torch.distributed as dist
    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def max_over_ranks(value: float) -> float:
    """The maximum of a per-rank scalar (e.g. a step time) over all ranks; the
    value itself when no process group is running."""
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier() -> None:
    import torch.distributed as dist
    if dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()


def job_throughput(units_per_rank: float, max_seconds: float, world_size: int) -> float:
    """Whole-job throughput when every rank processes units_per_rank units and the
    slowest rank takes max_seconds (weak scaling)."""
    return world_size * units_per_rank / max_seconds


def instance_cost(n: int, nparams: int, ngates: int | None = None) -> float:
    """Relative cost of one VQE instance on the batched engine: 2P+1 circuits,
    each ngates sweeps over 2^n amplitudes.  ngates defaults to the
    BasicEntangling ansatz at L = 4 (src/qml/vqc.rs:158-170): RY and RZ on every
    qubit plus an (n-1)-CNOT ladder per layer, 4(2n + n - 1) = 12n - 4 gates."""
    if ngates is None:
        ngates = 12 * n - 4
    return float((2 * nparams + 1) * ngates) * float(1 << n)


def shard_instances(costs, world_size: int, rank: int) -> list[int]:
    """Indices of the instances rank owns: longest-processing-time-first greedy
    assignment of the costs to world_size ranks (ties to the lower rank), the
    indices returned in ascending order.  Every instance goes to exactly one
    rank, and the same inputs give the same split on every rank."""
    if world_size < 1 or not 0 <= rank < world_size:
        raise ValueError("bad world size / rank")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world_size
    owner = [0] * len(costs)
    for i in order:
        r = min(range(world_size), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += costs[i]
    return [i for i in range(len(costs)) if owner[i] == rank]
