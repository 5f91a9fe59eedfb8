"""Multi-rank host logic of the benchmark on CPU: world_size 2 over gloo, each
rank with its own time; the job time is the max over ranks and the throughput
counts the work of both ranks (replicas, no data-path collective)."""
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
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parent.parent / "maquis-dmrg_b200"))
    from dmrgb200.replicas import job_throughput
    dist.init_process_group("gloo", rank=rank, world_size=world)
    dist.barrier()
    ms, rate = job_throughput(2.0 + rank, 1e9, world, dist)
    ms2, rate2 = job_throughput([1.0 + rank, 5.0 - rank], 1e9, world, dist)
    out[rank] = (ms, rate, ms2, rate2)
    dist.barrier()
    dist.destroy_process_group()


def test_job_throughput_two_ranks():
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
    for r in range(world):
        ms, rate, ms2, rate2 = out[r]
        assert ms == pytest.approx(3.0)
        assert rate == pytest.approx(2 * 1e9 / 3e-3)
        assert ms2 == [pytest.approx(2.0), pytest.approx(5.0)]
        assert rate2[1] == pytest.approx(2 * 1e9 / 5e-3)
