"""The multi-GPU bench path, exercised as two gloo ranks on CPU.

With N > 1 the bench runs one process per GPU (torchrun); registration pairs
are independent, so each rank registers its own pairs (replicas, no data-path
collective) and only the timing is combined: the job's time is the slowest
rank's (an all-reduce MAX), and the value is every rank's pairs over that
time.  This test runs those host steps in two processes over gloo: disjoint
pair seeds per rank, the MAX over ranks seen identically by both, the
whole-job rate, and the reference arm exiting at once on ranks other than 0.
"""
import json
import os
import socket

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, outdir):
    import datetime
    import sys
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    seeds = bench.pool_seeds(rank, 4)
    gathered = [None] * world
    dist.all_gather_object(gathered, seeds)
    local_ms = 10.0 + 5.0 * rank  # rank 1 is the slower one
    worst = bench.max_over_ranks(local_ms, dist, device="cpu")
    rate = bench.job_rate(world, 10, 16, worst)

    class Args:
        steps, warmup, gpus = 1, 0, world

    ref_rc = bench.run_reference(Args(), world, rank) if rank != 0 else None
    dist.barrier()
    dist.destroy_process_group()
    with open(os.path.join(outdir, f"rank{rank}.json"), "w") as f:
        json.dump({"seeds": gathered, "worst": worst, "rate": rate, "ref_rc": ref_rc}, f)


def test_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    s0, s1 = res[0]["seeds"]
    assert not set(s0) & set(s1)  # pairs are sharded: no pair on two ranks
    assert res[0]["seeds"] == res[1]["seeds"]
    assert res[0]["worst"] == res[1]["worst"] == 15.0  # the slowest rank's time, on every rank
    assert res[0]["rate"] == pytest.approx(2 * 10 * 16 / 15e-3)
    assert res[1]["ref_rc"] == 0  # the reference arm runs on rank 0 only
