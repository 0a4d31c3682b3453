"""Host logic of the multi-GPU path, on CPU: requests routed across ranks
(renderingengine_b200/routing.py), the job's time as the slowest rank's and
its work as every rank's, and per-request figures gathered to rank 0 --
exercised by two gloo ranks (the collectives are the same calls NCCL runs on
GPUs; the render path itself has no collective)."""
import json
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from renderingengine_b200 import routing as R
from renderingengine_b200 import workloads as W


def test_shard_requests_partitions_the_stream():
    work = [q.samples for q in W.request_stream(300)]
    for world in (1, 2, 3, 8):
        for policy in ("balanced", "round_robin"):
            shards = [R.shard_requests(work, world, r, policy) for r in range(world)]
            flat = sorted(i for s in shards for i in s)
            assert flat == list(range(len(work)))
            assert all(s == sorted(s) for s in shards)
            assert shards == [R.shard_requests(work, world, r, policy) for r in range(world)]  # deterministic
            if policy == "balanced" and world > 1:
                loads = [sum(work[i] for i in s) for s in shards]
                assert max(loads) - min(loads) <= max(work)
    with pytest.raises(ValueError):
        R.shard_requests(work, 2, 2)


def test_merge_served_combines_ranks():
    a = {"samples": 10, "first_arrival": 0.1, "last_completion": 2.0, "latencies": [1.0, 2.0]}
    b = {"samples": 30, "first_arrival": 0.0, "last_completion": 4.0, "latencies": [3.0]}
    m = R.merge_served([a, b])
    assert m["samples"] == 40 and m["makespan_s"] == 4.0 and m["samples_per_s"] == 10.0
    assert m["requests"] == 3 and m["latency_p50_s"] == 2.0


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        ms, units = R.max_time_sum_work(10.0 + rank, 100.0 * (rank + 1))
        work = [q.samples for q in W.request_stream(64)]
        mine = R.shard_requests(work, world, rank)
        part = {"samples": sum(work[i] for i in mine), "first_arrival": 0.0, "last_completion": 1.0 + rank,
                "latencies": [0.5 + rank] * len(mine), "ids": mine}
        parts = R.gather_to_rank0(part)
        if rank == 0:
            merged = R.merge_served(parts)
            ids = sorted(i for p in parts for i in p["ids"])
            with open(os.path.join(out_dir, "result.json"), "w") as f:
                json.dump({"ms": ms, "units": units, "merged": merged, "ids": ids, "n": len(work),
                           "total": sum(work)}, f)
        else:
            assert parts is None
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_route_and_reduce(tmp_path):
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    res = json.loads((tmp_path / "result.json").read_text())
    assert res["ms"] == 11.0 and res["units"] == 300.0
    assert res["ids"] == list(range(res["n"]))
    m = res["merged"]
    assert m["samples"] == res["total"] and m["makespan_s"] == 2.0 and m["requests"] == res["n"]
    assert m["latency_p99_s"] == 1.5 and np.isclose(m["samples_per_s"], res["total"] / 2.0)
