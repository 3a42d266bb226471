"""Distributed state vector: one n-qubit ket split over G = 2^g processes, one GPU each.

Quantum++ keeps a state in one process (its `ket` is an Eigen vector); this module is the
step beyond it for kets larger than one GPU's memory (31-34 qubits in complex128 on 2-16
B200s).

Layout. Physical qubit 0 is the most significant, as in qpp's big-endian order. Rank r holds
the 2^(n-g) amplitudes whose g most significant physical qubits spell r. Its local state is a
ket over physical qubits g..n-1, resident in HBM and driven by the library's kernels. A
logical -> physical map `perm` records where every logical qubit currently sits.

Gates. A gate whose physical targets are all local runs on the local state. A global target
first trades places with the most significant local qubit that the gate does not touch. Ranks r
and r ^ (1 << (g-1-p)) exchange the half of their local state in which that local qubit
differs from their own bit p: one send and one receive of 2^(n-g-1) amplitudes per rank (NCCL
over NVLink between GPUs), and the map records the swap. Global controls need no exchange: a
rank whose control bit is 0 skips the gate, the others apply it with the local controls only.
Norms and inner products are local reductions plus one all-reduce.

Communication goes through a `comm` object:
  * `TorchComm`: torch.distributed (NCCL on GPUs, gloo on CPUs), one process per rank;
  * `ThreadComm`: G ranks as threads of one process sharing one device, exchanging through
    device copies, so that the distributed algorithm can run where only one GPU is available.
    No kernel of one rank ever waits on another rank: every exchange is a host-synchronised copy.
"""
from __future__ import annotations

import threading

import numpy as np

from . import C128, C64, KET, State

__all__ = ["DistributedKet", "GpuLocal", "TorchComm", "ThreadComm", "ThreadHub"]


def _log2_exact(x):
    g = x.bit_length() - 1
    if x <= 0 or (1 << g) != x:
        raise ValueError(f"the number of ranks must be a power of two, got {x}")
    return g


# ---------------------------------------------------------------- transports
class TorchComm:
    """torch.distributed transport (one process per rank)."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self._dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)

    def sendrecv(self, sends, recvs, peer):
        """Send each tensor of `sends` to `peer` and receive `recvs` from it (same shapes,
        same order on both sides)."""
        dist = self._dist
        ops = []
        for s, r in zip(sends, recvs):
            ops.append(dist.P2POp(dist.isend, s, peer, self.group))
            ops.append(dist.P2POp(dist.irecv, r, peer, self.group))
        for w in dist.batch_isend_irecv(ops):
            w.wait()

    def allreduce_sum(self, x, like):
        import torch
        t = torch.tensor([x], dtype=torch.float64, device=like.device)
        self._dist.all_reduce(t, group=self.group)
        return float(t.item())

    def gather(self, t, root):
        """The ranks' tensors (same shape) on `root`, None elsewhere."""
        import torch
        out = [torch.empty_like(t) for _ in range(self.size)] if self.rank == root else None
        self._dist.gather(t, out, dst=root, group=self.group)
        return out

    def barrier(self):
        self._dist.barrier(group=self.group)


class ThreadHub:
    """Rendezvous of the ranks of a ThreadComm (one per emulated job)."""

    def __init__(self, size, timeout=60.0):
        self.size = size
        self.timeout = timeout
        self.bar = threading.Barrier(size, timeout=timeout)
        self.box = {}
        self.lock = threading.Lock()


class ThreadComm:
    """G ranks as threads of one process; exchanges are device (or host) copies between
    the ranks' tensors after a host barrier."""

    def __init__(self, hub, rank):
        self.hub = hub
        self.rank = rank
        self.size = hub.size

    def _sync_all(self):
        try:
            import torch
            if torch.cuda.is_available():
                torch.cuda.synchronize()
        except ImportError:
            pass

    def sendrecv(self, sends, recvs, peer):
        with self.hub.lock:
            self.hub.box[(self.rank, peer)] = sends
        self._sync_all()
        self.hub.bar.wait()
        src = self.hub.box[(peer, self.rank)]
        for r, s in zip(recvs, src):
            r.copy_(s)
        self._sync_all()
        self.hub.bar.wait()
        with self.hub.lock:
            self.hub.box.pop((self.rank, peer), None)

    def allreduce_sum(self, x, like=None):
        with self.hub.lock:
            self.hub.box[("sum", self.rank)] = x
        self.hub.bar.wait()
        total = sum(self.hub.box[("sum", r)] for r in range(self.size))
        self.hub.bar.wait()
        return total

    def gather(self, t, root):
        with self.hub.lock:
            self.hub.box[("gather", self.rank)] = t
        self._sync_all()
        self.hub.bar.wait()
        out = [self.hub.box[("gather", r)].clone() for r in range(self.size)] \
            if self.rank == root else None
        self._sync_all()
        self.hub.bar.wait()
        return out

    def barrier(self):
        self.hub.bar.wait()


# -------------------------------------------------------------- local states
class _DeviceArray:
    """A float view (2 reals per amplitude) of a state's device memory, for torch."""

    def __init__(self, ptr, n_reals, prec):
        self.__cuda_array_interface__ = {
            "shape": (n_reals,), "typestr": "<f8" if prec == C128 else "<f4",
            "data": (int(ptr), False), "version": 3, "strides": None}


class GpuLocal:
    """A rank's share of the ket: a resident qgpu ket over nl qubits."""

    def __init__(self, ctx, nl, prec=C128):
        self.ctx, self.nl, self.prec = ctx, nl, prec
        self.state = State(ctx, KET, [2] * nl, prec)

    def view(self):
        """torch float tensor aliasing the amplitudes (2 reals each)."""
        import torch
        return torch.as_tensor(_DeviceArray(self.state.device_ptr(), 2 << self.nl, self.prec),
                               device="cuda")

    def sync(self):
        self.ctx.synchronize()

    def apply(self, U, targets):
        self.state.apply(U, targets)

    def apply_ctrl(self, U, ctrl, targets):
        self.state.apply_ctrl(U, ctrl, targets)

    def norm2(self):
        return self.state.norm2()

    def scale(self, s):
        v = self.view()
        self.sync()
        v.mul_(s)
        import torch
        torch.cuda.synchronize()

    def upload(self, amps):
        self.state.upload(np.ascontiguousarray(amps, dtype=np.complex128))

    def numpy(self):
        return self.state.numpy()

    def free(self):
        self.state.free()


# ---------------------------------------------------------------- the ket
class DistributedKet:
    """An n-qubit ket over comm.size ranks (a power of two); `local` holds this rank's
    2^(n - g) amplitudes (GpuLocal on a GPU)."""

    def __init__(self, n, comm, local):
        self.n, self.comm = n, comm
        self.g = _log2_exact(comm.size)
        if n - self.g < 3:
            raise ValueError("each rank must hold at least 3 qubits")
        self.nl = n - self.g
        self.local = local
        self.perm = list(range(n))  # logical qubit -> physical qubit
        self.exchanges = 0

    # -- layout helpers
    def _bit(self, p):
        """This rank's value of global physical qubit p (< g)."""
        return (self.comm.rank >> (self.g - 1 - p)) & 1

    def _swap(self, p, l):
        """Global physical qubit p trades places with local physical qubit l."""
        a = self._bit(p)
        peer = self.comm.rank ^ (1 << (self.g - 1 - p))
        li = l - self.g
        blk = 1 << (self.nl - 1 - li)       # amplitudes per block
        nblk = 1 << li
        v = self.local.view()
        reals = 2 * blk
        # the blocks where local qubit li equals 1 - a go to the peer; the peer's blocks
        # where it equals a come back into the same places
        sends, recvs, places = [], [], []
        for j in range(nblk):
            start = 2 * (j * 2 * blk + (1 - a) * blk)
            seg = v[start:start + reals]
            sends.append(seg)
            recvs.append(seg.new_empty(seg.shape))
            places.append(seg)
        self.local.sync()
        self.comm.sendrecv(sends, recvs, peer)
        for dst, src in zip(places, recvs):
            dst.copy_(src)
        try:
            import torch
            if v.is_cuda:
                torch.cuda.synchronize()
        except ImportError:
            pass
        x = self.perm.index(p)
        y = self.perm.index(l)
        self.perm[x], self.perm[y] = l, p
        self.exchanges += 1

    def _localise(self, logical, keep=()):
        """Bring the physical positions of the logical qubits `logical` into the local part,
        never disturbing the physical positions in `keep`."""
        for q in logical:
            p = self.perm[q]
            if p >= self.g:
                continue
            busy = {self.perm[x] for x in logical} | set(keep)
            l = next(x for x in range(self.g, self.n) if x not in busy)
            self._swap(p, l)

    # -- ops
    def apply(self, U, targets):
        """qpp::apply(psi, U, targets) on the distributed ket (U is 2^k x 2^k, targets in
        U's order)."""
        self._localise(targets)
        self.local.apply(U, [self.perm[t] - self.g for t in targets])

    def apply_ctrl(self, U, ctrl, targets):
        """qpp::applyCTRL on qubits: U on the targets where every control is 1."""
        keep = [self.perm[c] for c in ctrl if self.perm[c] >= self.g]
        self._localise(targets, keep)
        for c in ctrl:
            p = self.perm[c]
            if p < self.g and self._bit(p) == 0:
                return  # this rank's amplitudes all have that control at 0
        local_ctrl = [self.perm[c] - self.g for c in ctrl if self.perm[c] >= self.g]
        lt = [self.perm[t] - self.g for t in targets]
        if local_ctrl:
            self.local.apply_ctrl(U, local_ctrl, lt)
        else:
            self.local.apply(U, lt)

    def norm2(self):
        like = self.local.view() if hasattr(self.local, "view") else None
        return self.comm.allreduce_sum(self.local.norm2(), like)

    def normalize(self):
        self.local.scale(1.0 / np.sqrt(self.norm2()))

    # -- host transfers (tests, small states)
    def scatter_from(self, psi):
        """Every rank passes the same full logical ket; each keeps its share (the layout
        is reset to the identity map)."""
        self.perm = list(range(self.n))
        D = 1 << self.nl
        r = self.comm.rank
        self.local.upload(np.asarray(psi, dtype=np.complex128)[r * D:(r + 1) * D])

    def gather_numpy(self, root=0):
        """The full logical ket on `root` (None elsewhere)."""
        self.local.sync()
        parts = self.comm.gather(self.local.view(), root)
        if parts is None:
            return None
        flat = np.concatenate([p.detach().cpu().numpy() for p in parts])
        phys = flat.view(np.complex128) if flat.dtype == np.float64 else \
            flat.view(np.complex64).astype(np.complex128)
        # physical axis i holds logical qubit perm^-1(i): move logical q to axis q
        a = phys.reshape([2] * self.n)
        return np.transpose(a, [self.perm[q] for q in range(self.n)]).reshape(-1)
