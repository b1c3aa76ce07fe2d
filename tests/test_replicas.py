"""The multi-GPU path's host logic on CPU: a world-size-2 gloo group runs the same replica plumbing
the benchmark runs over NCCL (barrier, max over ranks, whole-job rate, pooled latencies, the
round-robin request split), and the reference arm's non-leader ranks exit without work."""
import json
import os
import socket
import sys
import types

import pytest
import torch.multiprocessing as mp

from solidfem_b200 import workloads as W
from replicas import ReplicaGroup

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    group = ReplicaGroup.from_env("gloo", timeout_seconds=60)
    stream = W.serving_stream(count=37)
    share = group.shard(stream)
    # each rank "times" a different duration; the job ends with the slowest one
    seconds = 1.0 + rank
    group.barrier()
    result = {
        "rank": group.rank, "world": group.world, "leader": group.leader,
        "max": group.max(seconds), "sum": group.sum(rank + 1),
        "rate": group.rate(len(share), seconds),
        "ids": [r.index for r in share],
        "all_ids": group.gather([r.index for r in share]),
        "arrivals_sorted": all(a.arrival <= b.arrival for a, b in zip(share, share[1:])),
    }
    group.close()
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump(result, f)


def test_gloo_world_two(tmp_path):
    world = 2
    mp.start_processes(_worker, args=(world, free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    assert [r["rank"] for r in res] == [0, 1] and all(r["world"] == 2 for r in res)
    assert [r["leader"] for r in res] == [True, False]
    assert all(r["max"] == 2.0 and r["sum"] == 3.0 for r in res)
    # 37 requests over the slowest rank's 2 s, the same figure on every rank
    assert all(r["rate"] == pytest.approx(37 / 2.0) for r in res)
    a, b = set(res[0]["ids"]), set(res[1]["ids"])
    assert not (a & b) and a | b == set(range(37)) and len(a) == 19 and len(b) == 18
    assert all(r["all_ids"] == res[0]["ids"] + res[1]["ids"] for r in res)
    assert all(r["arrivals_sorted"] for r in res)


def test_single_process_group(monkeypatch):
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    g = ReplicaGroup.from_env("nccl")  # no process group, no device needed for one rank
    assert g.dist is None and g.world == 1 and g.leader
    assert g.max(2.5) == 2.5 and g.rate(3, 1.5) == 2.0
    assert g.gather([1, 2]) == [1, 2] and g.shard([5, 6, 7]) == [5, 6, 7]
    g.barrier()
    g.close()


def test_reference_arm_non_leader_exits_without_work(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench

    def fail(*a, **k):
        raise AssertionError("a non-leader rank ran the CPU sample")
    monkeypatch.setattr(bench, "oracle_solve", fail)
    monkeypatch.setattr(bench, "_oracle", fail)
    args = types.SimpleNamespace(warmup=3, steps=2, gpus=2)
    assert bench.run_reference(args, 1, 2) == 0
