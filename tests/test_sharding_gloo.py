"""Batched instances over several ranks on CPU: the greedy size-balanced
assignment, the generation of a rank's share, and the host gather of labels
(two gloo ranks on 127.0.0.1; no GPU, no NCCL)."""
import json
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _sizes(count=None):
    from gpu_hdbscan_b200 import synth
    return [n for n, _, _ in synth.batch_layout(synth.BATCH_WORKLOADS["batch_4096"], count)]


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_assignment_covers_every_instance_once_and_balances(world):
    from gpu_hdbscan_b200 import sharding
    sizes = _sizes()
    parts = sharding.assign_instances(sizes, world)
    assert len(parts) == world
    flat = [i for p in parts for i in p]
    assert sorted(flat) == list(range(len(sizes)))
    assert all(p == sorted(p) for p in parts)
    loads = sharding.rank_loads(sizes, parts)
    assert sum(loads) == sum(sizes)
    # greedy largest-first: the spread is at most one instance
    assert max(loads) - min(loads) <= max(sizes)
    # and the maximum is close to the even share here (many small instances)
    assert max(loads) <= sum(sizes) / world * 1.01 + 1
    assert parts == sharding.assign_instances(sizes, world)  # deterministic


def test_assignment_edge_cases():
    from gpu_hdbscan_b200 import sharding
    assert sharding.assign_instances([], 3) == [[], [], []]
    assert sharding.assign_instances([5, 5, 5], 4) == [[0], [1], [2], []]
    # ties go to the lower index and the lower rank
    assert sharding.assign_instances([3, 3, 3, 3], 2) == [[0, 2], [1, 3]]
    assert sharding.assign_instances([10, 1, 1, 1], 2) == [[0], [1, 2, 3]]
    with pytest.raises(ValueError):
        sharding.assign_instances([1], 0)


def test_a_ranks_share_is_generated_as_in_the_whole_batch():
    from gpu_hdbscan_b200 import sharding, synth
    bw = synth.BATCH_WORKLOADS["batch_4096"]
    count = 10
    full, layout = synth.generate_batch_torch(bw, device="cpu", count=count)
    parts = sharding.assign_instances([n for n, _, _ in layout], 2)
    for p in parts:
        views, sub = synth.generate_batch_torch(bw, device="cpu", count=count, indices=p)
        assert sub == [layout[i] for i in p]
        for v, i in zip(views, p):
            assert v.shape == full[i].shape
            assert (v == full[i]).all()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import torch
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench
    from gpu_hdbscan_b200 import sharding

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        sizes = [int(s) % 97 + 3 for s in _sizes(40)]  # small stand-in label arrays
        parts = sharding.assign_instances(sizes, world)
        # "labels" of instance i: i repeated, one per point
        local = [np.full(sizes[i], i, np.int32) for i in parts[rank]]
        got = sharding.gather_labels(local, parts, rank)
        total = bench.sum_over_ranks(len(parts[rank]), torch.device("cpu"))
        res = {"rank": rank, "total": total, "none_off_root": got is None}
        if rank == 0:
            res["ok"] = all(len(got[i]) == sizes[i] and (got[i] == i).all()
                            for i in range(len(sizes)))
            res["count"] = len(got)
        dist.barrier()
    finally:
        dist.destroy_process_group()
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump(res, f)


def test_two_gloo_ranks_gather_every_instances_labels(tmp_path):
    world = 2
    ctx = mp.get_context("spawn")
    port = free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, str(tmp_path)))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0, f"rank exited with {p.exitcode}"
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    assert res[0]["ok"] and res[0]["count"] == 40
    assert not res[0]["none_off_root"] and res[1]["none_off_root"]
    assert res[0]["total"] == res[1]["total"] == 40
