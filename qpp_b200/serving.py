"""Serving loop front-end and the synthetic serving workload.

`Server` wraps qgpu_server_* (include/qpp_b200.h): a C++ worker thread that
drains a request queue either with continuous batching (mode BATCHED: every
request that arrived while the previous launch ran joins the next
trajectory-kernel launch; density matrices and registers above 20 qubits run
on the resident engine on a second stream) or one request at a time on the
resident engine in complex128 (mode PLAIN).

`request_pool` builds the synthetic request mix of the serving benchmark
(seeded): 90% kets of 12-28 qubits with P(n) proportional to 2^-(n-12),
layered circuits of depth U{10..60} (a Haar 1-qubit gate on every qubit,
then Haar 2-qubit gates on a random perfect matching), depolarising noise
p = 1e-3 per qubit per step sampled by trajectories, log-uniform shot counts
in 1..1000, 20% of them with mid-circuit Z measurements of 1-3 random qubits;
10% density matrices of 8-13 qubits with the 2-qubit channel (depolarising
p = 0.01 composed with amplitude damping gamma = 0.02 on each qubit, 16
Kraus operators) after every 2-qubit gate.
"""
from __future__ import annotations

import ctypes as ct
import math
import threading
import time

import numpy as np

from . import C64, KET, RHO, Circuit, check, lib, vp
from .workloads import haar_unitary

BATCHED, PLAIN = 0, 1


class Server:
    def __init__(self, device=0, hbm_budget=180 * 2 ** 30, mode=BATCHED):
        self.h = vp()
        check(lib().qgpu_server_create(ct.c_int(device), ct.c_uint64(int(hbm_budget)),
                                       ct.c_int(mode), ct.byref(self.h)))
        self.mode = mode

    def submit(self, circuit, kind, p, shots, seed):
        rid = ct.c_uint64()
        check(lib().qgpu_server_submit(self.h, circuit.h, ct.c_int(kind), ct.c_double(p),
                                       ct.c_uint64(shots), ct.c_uint64(seed), ct.byref(rid)))
        return rid.value

    def wait(self, rid, shots=0, nc=1, timeout=-1.0):
        lat = ct.c_double()
        samples = np.zeros(max(shots, 1), dtype=np.uint64) if shots else None
        dits = np.zeros(max(shots * max(nc, 1), 1), dtype=np.uint32) if shots else None
        check(lib().qgpu_server_wait(
            self.h, ct.c_uint64(rid), ct.c_double(timeout), ct.byref(lat),
            None if samples is None else samples.ctypes.data_as(ct.c_void_p),
            None if dits is None else dits.ctypes.data_as(ct.c_void_p)))
        return lat.value, samples, dits

    def stats(self):
        b, t, e, busy = ct.c_uint64(), ct.c_uint64(), ct.c_uint64(), ct.c_double()
        check(lib().qgpu_server_stats(self.h, ct.byref(b), ct.byref(t), ct.byref(e),
                                      ct.byref(busy)))
        return {"batches": b.value, "trajectories": t.value, "engine_runs": e.value,
                "busy_s": busy.value}

    def close(self):
        if self.h:
            check(lib().qgpu_server_destroy(self.h))
            self.h = None


def _depol(p):
    I2 = np.eye(2, dtype=np.complex128)
    X = np.array([[0, 1], [1, 0]], dtype=np.complex128)
    Y = np.array([[0, -1j], [1j, 0]], dtype=np.complex128)
    Z = np.diag([1, -1]).astype(np.complex128)
    return [math.sqrt(1 - p) * I2] + [math.sqrt(p / 3) * P for P in (X, Y, Z)]


def _amp_damp(g):
    return [np.array([[1, 0], [0, math.sqrt(1 - g)]], dtype=np.complex128),
            np.array([[0, math.sqrt(g)], [0, 0]], dtype=np.complex128)]


def minimal_kraus(Ks, tol=1e-14):
    """The same channel with the fewest Kraus operators: eigenvectors of the
    Choi matrix sum_i vec(K_i) vec(K_i)^+ scaled by sqrt(eigenvalue)."""
    d = Ks[0].shape[0]
    C = sum(np.outer(K.reshape(-1, order="F"), K.reshape(-1, order="F").conj()) for K in Ks)
    w, V = np.linalg.eigh((C + C.conj().T) / 2)
    return [np.sqrt(w[i]) * V[:, i].reshape((d, d), order="F")
            for i in range(len(w)) if w[i] > tol * max(w.max(), 1)]


def pair_channel():
    """(depolarising p=0.01 o amplitude damping gamma=0.02) on each qubit of
    a pair: the 8 composed single-qubit products reduce (Choi rank) to 4
    operators per qubit, so the pair channel has 4 x 4 = 16 Kraus operators."""
    one = minimal_kraus([D @ A for D in _depol(0.01) for A in _amp_damp(0.02)])
    return [np.kron(a, b) for a in one for b in one]


class Request:
    """A request template; `steps` lists its circuit as ("gate", U, targets),
    ("channel", Ks, targets) and ("measure", [q], dit, destructive) tuples."""
    __slots__ = ("circuit", "kind", "n", "p", "shots", "nc", "steps")

    def __init__(self, circuit, kind, n, p, shots, nc, steps=None):
        self.circuit, self.kind, self.n, self.p, self.shots, self.nc = \
            circuit, kind, n, p, shots, nc
        self.steps = steps if steps is not None else []


def request_pool(count, seed=2025, max_ket_qubits=28, max_rho_qubits=13):
    """`count` request templates of the serving mix (see module docstring)."""
    rng = np.random.default_rng(seed)
    bank1 = [haar_unitary(rng, 2) for _ in range(128)]
    bank2 = [haar_unitary(rng, 4) for _ in range(128)]
    chan = pair_channel()
    ns = np.arange(12, max_ket_qubits + 1)
    pn = 2.0 ** -(ns - 12)
    pn /= pn.sum()
    pool = []
    for _ in range(count):
        kind = KET if rng.random() < 0.9 else RHO
        n = int(rng.choice(ns, p=pn)) if kind == KET else int(rng.integers(8, max_rho_qubits + 1))
        depth = int(rng.integers(10, 61))
        measure = kind == KET and rng.random() < 0.2
        meas_layers = set(int(x) for x in rng.choice(depth, size=min(2, depth), replace=False)) \
            if measure else set()
        nc = 6 if measure else 1
        c = Circuit(n, 2, nc)
        steps = []
        creg = 0
        for layer in range(depth):
            for q in range(n):
                U = bank1[int(rng.integers(128))]
                c.gate(U, [q])
                steps.append(("gate", U, [q]))
            perm = rng.permutation(n)
            for i in range(n // 2):
                a, b = int(perm[2 * i]), int(perm[2 * i + 1])
                U = bank2[int(rng.integers(128))]
                c.gate(U, [a, b])
                steps.append(("gate", U, [a, b]))
                if kind == RHO:
                    c_channel(c, chan, [a, b])
                    steps.append(("channel", chan, [a, b]))
            if layer in meas_layers:
                k = int(rng.integers(1, 4))
                for q in rng.choice(n, size=k, replace=False):
                    if creg < nc:
                        c.measure([int(q)], creg, destructive=False)
                        steps.append(("measure", [int(q)], creg, False))
                        creg += 1
        shots = int(round(math.exp(rng.uniform(0, math.log(1000)))))
        pool.append(Request(c, kind, n, 1e-3 if kind == KET else 0.0, max(shots, 1), nc, steps))
    return pool


def c_channel(c, Ks, target):
    Ks = [np.asfortranarray(np.asarray(K, dtype=np.complex128)) for K in Ks]
    packed = np.ascontiguousarray(np.concatenate([K.reshape(-1, order="F") for K in Ks]))
    t = np.ascontiguousarray(np.asarray(target, dtype=np.uint64))
    check(lib().qgpu_circuit_channel(c.h, packed.ctypes.data_as(ct.POINTER(ct.c_double)),
                                     ct.c_uint32(len(Ks)), ct.c_uint64(Ks[0].shape[0]),
                                     t.ctypes.data_as(ct.POINTER(ct.c_uint64)),
                                     ct.c_uint32(len(target))))


def run_open_loop(server, pool, rate, duration, seed=7, max_requests=None):
    """Poisson arrivals at `rate` req/s for `duration` s (requests cycle
    through `pool`). Returns latencies (s), completed count and the wall time
    from the first arrival to the last completion."""
    rng = np.random.default_rng(seed)
    arrivals = []
    t = 0.0
    while t < duration:
        t += rng.exponential(1.0 / rate)
        arrivals.append(t)
        if max_requests and len(arrivals) >= max_requests:
            break
    ids = []
    lock = threading.Lock()
    lat = []

    def waiter():
        i = 0
        while True:
            with lock:
                if i >= len(ids) and done_submitting[0]:
                    return
                if i >= len(ids):
                    rid = None
                else:
                    rid, req = ids[i]
            if rid is None:
                time.sleep(0.0005)
                continue
            lt, _, _ = server.wait(rid)
            lat.append(lt)
            i += 1

    done_submitting = [False]
    w = threading.Thread(target=waiter)
    w.start()
    t0 = time.perf_counter()
    for k, ta in enumerate(arrivals):
        now = time.perf_counter() - t0
        if ta > now:
            time.sleep(ta - now)
        req = pool[k % len(pool)]
        rid = server.submit(req.circuit, req.kind, req.p, req.shots, seed=1000 + k)
        with lock:
            ids.append((rid, req))
    with lock:
        done_submitting[0] = True
    w.join()
    wall = time.perf_counter() - t0
    return np.array(lat), len(lat), wall


def summarize(lat, completed, wall):
    return {"completed": int(completed), "circuits_per_s": completed / wall if wall > 0 else 0.0,
            "p50_ms": float(np.percentile(lat, 50) * 1e3) if len(lat) else None,
            "p99_ms": float(np.percentile(lat, 99) * 1e3) if len(lat) else None,
            "wall_s": wall}
