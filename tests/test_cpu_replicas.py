"""The multi-replica bench path on CPU: two ranks over gloo use the bench's
own barrier and max-over-ranks helpers, and the reference arm does no work
on ranks other than 0.  (On the GPU box the same helpers run over NCCL, one
replica per GPU, with no collective on the data path.)"""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch
    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world,
                                         timeout=datetime.timedelta(seconds=60))
    try:
        assert bench.dist_env() == (rank, rank, world)
        barrier, max_over_ranks = bench.rank_reducers(world, "cpu")
        barrier()
        # each replica reports its own ms/step; the run reports the slowest
        out[rank] = max_over_ranks(10.0 + 5.0 * rank)
        barrier()
    finally:
        torch.distributed.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank_main, args=(world, _free_port(), out), nprocs=world, start_method="spawn", join=True)
    assert dict(out) == {0: 15.0, 1: 15.0}


def test_single_rank_reducers_pass_through():
    sys.path.insert(0, ROOT)
    import bench
    barrier, max_over_ranks = bench.rank_reducers(1, "cpu")
    barrier()
    assert max_over_ranks(3.5) == 3.5


def test_reference_arm_idle_on_other_ranks(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    # rank 1 returns before importing or running anything of the reference
    assert bench.run_reference(None) is None


def test_bench_launches_its_own_replicas():
    """`bench.py --gpus 2` outside a launcher starts two ranks itself (the
    same torch.distributed.run command the GPU run uses); the replica-check
    mode does only the rank plumbing, over gloo on CPU."""
    import json
    import subprocess
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "replica-check", "--gpus", "2"],
                       capture_output=True, text=True, timeout=240, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    assert json.loads(lines[0]) == {"impl": "replica-check", "n_ranks": 2, "max_over_ranks": 2.0}


def test_bench_refuses_more_gpus_than_visible():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.launch_replicas(4, ["--steps", "1"], visible_gpus=1) == 2
