"""The N>1 benchmark path on CPU: two gloo ranks (127.0.0.1) run the replica bookkeeping
that bench.py runs over NCCL -- slowest-rank timing and whole-job throughput -- and the
reference arm's rank rule (only rank 0 runs and prints)."""
import contextlib
import io
import json
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist

    from tensorfim_b200 import replicas
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        my_ms = [3.0, 5.5][rank]                       # rank 1 is the slowest
        ms = replicas.max_over_ranks(my_ms)
        value = replicas.job_throughput(1_000_000, ms)
        with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
            json.dump({"world": replicas.world_size(), "ms": ms, "value": value}, f)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_slowest_rank(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    res = [json.load(open(tmp_path / f"r{r}.json")) for r in range(world)]
    for r in res:
        assert r["world"] == 2
        assert r["ms"] == 5.5
        assert r["value"] == pytest.approx(2 * 1_000_000 / 5.5e-3)
    assert res[0] == res[1]


def test_single_process_is_identity():
    from tensorfim_b200 import replicas
    assert replicas.world_size() == 1
    assert replicas.max_over_ranks(4.25) == 4.25
    assert replicas.job_throughput(100, 2.0) == pytest.approx(50_000.0)


def test_reference_arm_runs_on_rank_zero_only():
    import argparse

    import bench
    args = argparse.Namespace(workload="cfg1", ref_scale=0.02, steps=1, warmup=0)
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        assert bench.run_reference_arm(args, rank=1, world=2) == 0
    assert buf.getvalue() == ""
