"""The bench's N-GPU path on the CPU: world_size-2 gloo ranks (127.0.0.1) take the slowest
rank's time and report whole-job replica throughput; under torchrun the reference arm runs
on rank 0 only. The river path has no exchange step, so replicas share nothing else."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ms = bench.max_over_ranks(10.0 + 5.0 * rank, world, torch.device("cpu"))
    out[rank] = (ms, bench.replica_rate(1000.0, world, ms / 1e3))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_and_replica_rate():
    port = _free_port()
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for rank in range(world):
        ms, rate = res[rank]
        assert ms == 15.0
        assert rate == pytest.approx(2 * 1000.0 / 0.015)


def test_reference_arm_prints_on_rank_zero_only(monkeypatch, capsys):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    class Args:
        steps, warmup, gpus = 1, 0, 2
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    assert bench.run_reference(Args()) == 0
    assert capsys.readouterr().out == ""
