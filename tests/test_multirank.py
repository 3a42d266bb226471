"""N > 1 path on CPU: two gloo ranks run the bench's cross-rank reduction
(replicas: job time = slowest rank, job work = sum over ranks) and the
reference arm's rank gating, without a GPU."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import sys
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ms, total = bench.reduce_over_ranks(dist, 10.0 + 5 * rank, 1000 * (rank + 1))
    out[rank] = (ms, total)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_reduction_gloo():
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, port, out), nprocs=world, start_method="spawn")
    assert out[0] == out[1] == (15.0, 3000.0)


def test_reference_arm_other_ranks_exit_without_work(monkeypatch):
    import bench
    monkeypatch.setenv("RANK", "1")

    class A:
        qubits = 30
        steps = 40
        warmup = 3
        gpus = 2

    assert bench.run_reference(A()) == 0
