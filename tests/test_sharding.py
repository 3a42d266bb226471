"""Instance sharding across GPUs (qpp_b200.sharding), on the CPU: the
placement by free HBM respects every device's memory and fills devices in
proportion to it; two gloo ranks with different free memory compute the same
placement and split the instances between them exactly once; the multi-GPU
serving front routes requests by outstanding work (a stand-in server class
records the calls, no GPU)."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from qpp_b200 import sharding


def test_assign_respects_memory_and_balances():
    sizes = [2 ** k for k in (10, 12, 14, 16, 18, 20, 22) for _ in range(9)]
    free = [2 ** 26, 2 ** 27]  # the second device has twice the room
    place = sharding.assign(sizes, free)
    load = [0, 0]
    for s, d in zip(sizes, place):
        load[d] += s
    assert all(load[d] <= free[d] for d in range(2))
    assert abs(load[1] / load[0] - 2) < 0.25
    with pytest.raises(MemoryError):
        sharding.assign([2 ** 30], free)
    # deterministic: the same inputs give the same placement
    assert sharding.assign(sizes, free) == place


def test_instance_bytes():
    assert sharding.instance_bytes(True, 20, 16) == 16 * 2 ** 20
    assert sharding.instance_bytes(False, 10, 8) == 8 * 4 ** 10


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
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from qpp_b200 import sharding as sh
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sizes = [(i * 7919) % 5000 + 100 for i in range(300)]
    mine = sh.shard_for_rank(sizes, free_local=10 ** 6 * (rank + 1), dist=dist)
    out[rank] = mine
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_split_instances_once():
    world = 2
    port = _free_port()
    out = mp.get_context("spawn").Manager().dict()
    mp.start_processes(_worker, args=(world, port, out), nprocs=world, start_method="spawn")
    a, b = set(out[0]), set(out[1])
    assert not (a & b) and a | b == set(range(300))
    sizes = [(i * 7919) % 5000 + 100 for i in range(300)]
    ba, bb = sum(sizes[i] for i in a), sum(sizes[i] for i in b)
    assert bb > ba  # rank 1 reported twice the free memory


class _FakeServer:
    def __init__(self, device, budget, mode):
        self.device, self.n, self.closed = device, 0, False

    def submit(self, circuit, kind, p, shots, seed):
        self.n += 1
        return self.n

    def wait(self, rid, shots=0, nc=1, timeout=-1.0):
        return 0.0, None, None

    def close(self):
        self.closed = True


class _Circ:
    def __init__(self, nq):
        self.nq = nq


def test_multiserver_routes_by_outstanding_work():
    from qpp_b200 import KET
    ms = sharding.MultiServer([0, 1], hbm_budget=2 ** 40, server_cls=_FakeServer)
    big = ms.submit(_Circ(20), KET, 1e-3, 1000, 1)        # device 0 takes the big one
    smalls = [ms.submit(_Circ(12), KET, 1e-3, 10, 2 + k) for k in range(5)]
    assert ms.device_of(big) == 0
    assert all(ms.device_of(m) == 1 for m in smalls)     # the rest go to the idle device
    ms.wait(big)
    assert ms.work[0] == 0 and ms.held[0] == 0
    nxt = ms.submit(_Circ(12), KET, 1e-3, 10, 9)
    assert ms.device_of(nxt) == 0                         # device 0 is free again
    ms.close()
    assert all(s.closed for s in ms.servers)
