"""Seeded synthetic workloads of the benchmark configurations.

The reference draws its inputs from an unseeded mt19937 (include/qpp/
random.hpp:257-412), so every input here comes from this project's own
seeded generator and is fed identically to the GPU path and to the CPU
baseline:

  haar_unitary   QR of a complex Ginibre matrix with R's diagonal phases
                 moved into Q (Mezzadri, Notices AMS 54, 2007).
  layered_circuit(n, depth)  each layer: a Haar 1-qubit gate on every qubit,
                 then a Haar 2-qubit gate on each pair of a uniformly random
                 perfect matching (n // 2 pairs).
  ket_gate_sequence(n)       1000 gates, 70% Haar 2x2 on a uniform target and
                 30% Haar 4x4 on a uniform ordered pair, then 100 controlled
                 Haar 2x2 with 1-3 distinct controls.
"""
from __future__ import annotations

import numpy as np


def haar_unitary(rng, D):
    Z = (rng.standard_normal((D, D)) + 1j * rng.standard_normal((D, D))) / np.sqrt(2)
    Q, R = np.linalg.qr(Z)
    d = np.diag(R)
    return (Q * (d / np.abs(d))).astype(np.complex128)


def layered_circuit(n, depth, seed):
    """List of `depth` layers; a layer is a list of (U, targets)."""
    rng = np.random.default_rng(seed)
    layers = []
    for _ in range(depth):
        gates = [(haar_unitary(rng, 2), [q]) for q in range(n)]
        perm = rng.permutation(n)
        for i in range(n // 2):
            gates.append((haar_unitary(rng, 4), [int(perm[2 * i]), int(perm[2 * i + 1])]))
        layers.append(gates)
    return layers


def ket_gate_sequence(n, seed, n_gates=1000, n_ctrl=100):
    """[(U, ctrl, targets)] with ctrl == [] for plain gates."""
    rng = np.random.default_rng(seed)
    seq = []
    for _ in range(n_gates):
        if rng.random() < 0.7:
            t = [int(rng.integers(n))]
        else:
            t = [int(x) for x in rng.choice(n, size=2, replace=False)]
        seq.append((haar_unitary(rng, 2 ** len(t)), [], t))
    for _ in range(n_ctrl):
        nc = int(rng.integers(1, 4))
        sub = [int(x) for x in rng.choice(n, size=nc + 1, replace=False)]
        seq.append((haar_unitary(rng, 2), sub[:nc], sub[nc:]))
    return seq


def gate_bytes(n, elem_bytes=16, n_ctrl=0):
    """Algorithmic bytes of one gate on an n-qubit ket: every touched
    amplitude is read once and written once."""
    return 2 * elem_bytes * (2 ** (n - n_ctrl))
