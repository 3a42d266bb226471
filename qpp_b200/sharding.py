"""Instance sharding across GPUs: independent instances (batched circuits) or
requests (serving) placed on devices by free HBM, one process or one server
per GPU, no communication on the data path.

Quantum++ runs every state in one process; independent states only need a
placement. `assign(sizes, free)` places instances of `sizes` bytes on devices
with `free` bytes each: largest first (longest-processing-time order), each to
the device whose assigned bytes relative to its free memory are lowest among
those where it still fits, so the devices fill in proportion to their free
HBM. The placement is a pure function of its inputs, so every rank of a job
computes the same one (`shard_for_rank` gathers the ranks' free memory first)
and each rank runs only its own instances.

`MultiServer` is the serving loop over several GPUs: one `serving.Server` per
device, each request routed to the device with the least outstanding work
(state bytes x shots) among those whose HBM budget still holds it.
"""
from __future__ import annotations

import threading

__all__ = ["assign", "shard_for_rank", "instance_bytes", "MultiServer"]


def instance_bytes(kind_is_ket, n_qubits, elem_bytes):
    """HBM bytes of one instance's state: 2^n amplitudes (ket) or 4^n
    elements (density matrix) of elem_bytes each."""
    return (1 << n_qubits if kind_is_ket else 1 << (2 * n_qubits)) * elem_bytes


def assign(sizes, free):
    """Device index of every instance: longest-first, each to the device with
    the lowest (assigned + size) / free among those with room. Raises
    MemoryError when an instance fits on no device."""
    nd = len(free)
    if nd == 0:
        raise ValueError("no devices")
    load = [0] * nd
    out = [-1] * len(sizes)
    for i in sorted(range(len(sizes)), key=lambda k: (-sizes[k], k)):
        best, best_key = -1, None
        for d in range(nd):
            if load[d] + sizes[i] > free[d]:
                continue
            key = ((load[d] + sizes[i]) / free[d], d)
            if best_key is None or key < best_key:
                best, best_key = d, key
        if best < 0:
            raise MemoryError(f"instance {i} ({sizes[i]} bytes) fits on no device")
        out[i] = best
        load[best] += sizes[i]
    return out


def shard_for_rank(sizes, free_local, dist=None):
    """The instances this rank runs: every rank contributes its free HBM
    (all_gather), all compute the same `assign`, each keeps its own."""
    if dist is None or not dist.is_initialized():
        return list(range(len(sizes)))
    import torch
    world, rank = dist.get_world_size(), dist.get_rank()
    backend = dist.get_backend()
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else "cpu"
    t = torch.tensor([float(free_local)], dtype=torch.float64, device=dev)
    parts = [torch.zeros_like(t) for _ in range(world)]
    dist.all_gather(parts, t)
    free = [float(p.item()) for p in parts]
    placement = assign(sizes, free)
    return [i for i, d in enumerate(placement) if d == rank]


class MultiServer:
    """The serving loop over several GPUs: `serving.Server` per device,
    requests routed by outstanding work within each device's HBM budget."""

    def __init__(self, devices, hbm_budget=180 * 2 ** 30, mode=0, server_cls=None):
        if server_cls is None:
            from .serving import Server as server_cls
        self.devices = list(devices)
        self.budget = hbm_budget
        self.servers = [server_cls(d, hbm_budget, mode) for d in self.devices]
        self.lock = threading.Lock()
        self.work = [0] * len(self.servers)    # outstanding state bytes x shots
        self.held = [0] * len(self.servers)    # outstanding state bytes
        self.where = {}                        # request id -> (server, work, bytes)
        self.next_id = 1

    def _pick(self, nbytes, cost):
        best, best_key = -1, None
        for d in range(len(self.servers)):
            if self.held[d] + nbytes > self.budget and self.held[d] > 0:
                continue
            key = (self.work[d] + cost, d)
            if best_key is None or key < best_key:
                best, best_key = d, key
        return best if best >= 0 else min(range(len(self.servers)), key=lambda d: self.held[d])

    def submit(self, circuit, kind, p, shots, seed, n_qubits=None, elem_bytes=8):
        from . import KET
        n = circuit.nq if n_qubits is None else n_qubits
        nbytes = instance_bytes(kind == KET, n, elem_bytes)
        cost = nbytes * (shots if kind == KET else 1)
        with self.lock:
            d = self._pick(nbytes, cost)
            self.work[d] += cost
            self.held[d] += nbytes
            rid = self.servers[d].submit(circuit, kind, p, shots, seed)
            mid = self.next_id
            self.next_id += 1
            self.where[mid] = (d, rid, cost, nbytes)
        return mid

    def wait(self, mid, shots=0, nc=1, timeout=-1.0):
        from . import Timeout
        with self.lock:
            d, rid, cost, nbytes = self.where[mid]
        try:
            out = self.servers[d].wait(rid, shots, nc, timeout)
        except Timeout:
            raise  # still pending on its device: keep it counted
        except BaseException:
            self._release(mid, d, cost, nbytes)
            raise
        self._release(mid, d, cost, nbytes)
        return out

    def _release(self, mid, d, cost, nbytes):
        with self.lock:
            self.where.pop(mid, None)
            self.work[d] -= cost
            self.held[d] -= nbytes

    def device_of(self, mid):
        with self.lock:
            return self.devices[self.where[mid][0]]

    def close(self):
        for s in self.servers:
            s.close()
