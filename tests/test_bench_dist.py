"""bench.py's multi-rank path on CPU: world_size-2 gloo ranks agree on the
job time (max over ranks), compute whole-job throughput, and the reference
arm runs on rank 0 only."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    ms = 10.0 * (rank + 1)  # rank 1 is the slow one
    job_ms = bench.max_over_ranks(ms)
    dist.barrier()
    dist.destroy_process_group()
    out[rank] = (job_ms, bench.job_mpts(world, 2_000_000, job_ms), bench.dist_env())


def test_two_gloo_ranks_take_the_max():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank_main, args=(world, port, out), nprocs=world, join=True,
                           start_method="spawn")
        res = dict(out)
    assert res[0][0] == res[1][0] == 20.0
    # 2 replicas x 2M points in 20 ms = 200 Mpoints/s
    assert res[0][1] == pytest.approx(200.0)
    assert res[1][2] == (2, 1, 1)


def test_single_process_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5) == 3.5
    assert bench.job_mpts(1, 1_000_000, 1.0) == pytest.approx(1000.0)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")

    class Args:
        steps, warmup, gpus = 1, 1, 2
    bench.run_reference(Args())  # returns at once: no work, no output on rank 1
    assert capsys.readouterr().out == ""
