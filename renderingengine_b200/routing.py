"""Host routing of render requests across GPUs (one process per GPU).

Nothing on the render path crosses GPUs: pixels, views and requests are
independent, so several GPUs run as replicas, each with its own render
server, and a host-side router decides which rank serves which request.
Results and latencies come back to rank 0 over the process group
(`torch.distributed`, NCCL or gloo); the only collectives are these small
host-side reductions, never a data-path exchange.
"""
from __future__ import annotations

import heapq
from typing import Sequence


def shard_requests(work: Sequence[float], world: int, rank: int, policy: str = "balanced") -> list[int]:
    """Indices of the requests rank `rank` of `world` serves, in arrival
    order.  `work[i]` is request i's estimated cost (pixels x samples).
    "round_robin": request i goes to rank i % world.  "balanced": requests,
    in arrival order, go to the rank with the least work assigned so far
    (lowest rank on ties), so every rank sees the same deterministic plan."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    if policy == "round_robin":
        return [i for i in range(len(work)) if i % world == rank]
    if policy != "balanced":
        raise ValueError(f"unknown routing policy {policy!r}")
    heap = [(0.0, r) for r in range(world)]
    mine = []
    for i, w in enumerate(work):
        load, r = heapq.heappop(heap)
        if r == rank:
            mine.append(i)
        heapq.heappush(heap, (load + float(w), r))
    return mine


def max_time_sum_work(ms: float, units: float, group=None) -> tuple[float, float]:
    """(max over ranks of `ms`, sum over ranks of `units`): the job's time
    is its slowest rank's, its work every rank's."""
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return float(ms), float(units)
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    u = torch.tensor([units], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    dist.all_reduce(u, op=dist.ReduceOp.SUM, group=group)
    return float(t.item()), float(u.item())


def gather_to_rank0(obj, group=None):
    """Every rank's `obj` as a list on rank 0 (None elsewhere)."""
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return [obj]
    out = [None] * dist.get_world_size(group) if dist.get_rank(group) == 0 else None
    dist.gather_object(obj, out, dst=0, group=group)
    return out


def merge_served(parts: list[dict]) -> dict:
    """Job-level figures of a routed stream from the ranks' parts (each with
    `samples`, `first_arrival`, `last_completion`, `latencies`): samples/s
    over the span from the first arrival to the last completion anywhere,
    latency percentiles over every request."""
    import numpy as np
    samples = sum(p["samples"] for p in parts)
    first = min(p["first_arrival"] for p in parts)
    last = max(p["last_completion"] for p in parts)
    lat = np.concatenate([np.asarray(p["latencies"], np.float64) for p in parts])
    span = last - first
    return {"samples": samples, "makespan_s": span, "samples_per_s": samples / span if span > 0 else 0.0,
            "latency_p50_s": float(np.percentile(lat, 50)), "latency_p99_s": float(np.percentile(lat, 99)),
            "latency_mean_s": float(lat.mean()), "requests": int(lat.size)}
