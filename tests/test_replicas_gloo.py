"""The multi-GPU path is replicas only: each rank runs its own copy of the
workload and the bench reports the whole job's throughput timed by the
slowest rank.  Two gloo ranks on CPU check the reduction and the value, and
that the reference arm runs on rank 0 only."""
import os
import socket

import pytest
import torch.multiprocessing as mp

import bench


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = [120.0, 150.0][rank]
        m = bench.max_over_ranks(ms, dist, device="cpu")
        out[rank] = (m, bench.whole_job_value(world, 8_000_000, 1000, 5, m))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_max_and_whole_job_value():
    port = _free_port()
    with mp.get_context("spawn").Manager() as man:
        out = man.dict()
        mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    assert res[0][0] == res[1][0] == 150.0
    # 2 replicas x 8e6 cells x 1000 steps x 5 runs in 150 ms
    assert res[0][1] == pytest.approx(2 * 8e6 * 1000 * 5 / 0.150 / 1e9)


def test_single_process_reduction_is_identity():
    assert bench.max_over_ranks(3.5, None) == 3.5


def test_reference_arm_runs_on_rank_zero_only(capsys):
    class A:
        config, steps, warmup = "config2", 1, 3
    assert bench.run_reference(A(), rank=1, world=2) == 0
    assert capsys.readouterr().out == ""
