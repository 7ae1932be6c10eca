"""The multi-GPU path of bench.py on CPU: N independent replicas, one process
per rank, only the timing reduced across ranks (max over ranks).  Runs as two
gloo ranks on 127.0.0.1; no GPU, no NCCL."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import torch
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench
    from gpu_hdbscan_b200 import synth

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        # each rank "measures" its own duration; every rank must see the max
        ms = 10.0 * (rank + 1) + 0.25
        got = bench.max_over_ranks(ms, torch.device("cpu"))
        w = bench.replica_workload(synth.WORKLOADS["blobs_100k_d12"], rank)
        X = synth.sample(w, 64)
        res = {"rank": rank, "max_ms": got, "seed": w.seed, "n": w.n,
               "x0": [float(v) for v in X[0]],
               "rate": bench.whole_job_rate(w.n, 3, world, got)}
        dist.barrier()
    finally:
        dist.destroy_process_group()
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump(res, f)


def test_two_gloo_ranks_reduce_timing_and_seed_replicas(tmp_path):
    world = 2
    ctx = mp.get_context("spawn")
    port = free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0, f"rank exited with {p.exitcode}"
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    # the max over ranks, seen identically by every rank
    assert res[0]["max_ms"] == res[1]["max_ms"] == 20.25
    # distinct seeded replicas of the same workload
    assert res[0]["seed"] != res[1]["seed"]
    assert res[0]["n"] == res[1]["n"]
    assert res[0]["x0"] != res[1]["x0"]
    # whole-job rate: world replicas x n points x steps over the slowest rank's time
    assert res[0]["rate"] == pytest.approx(2 * 100_000 * 3 / 0.02025)


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "3",
                        "--workload", "blobs_100k_d12"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
