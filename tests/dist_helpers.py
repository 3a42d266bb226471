"""Shared pieces of the distributed-ket tests: a host-memory local backend (numpy,
through the oracle's apply) and a seeded random circuit with its full-state oracle result."""
import numpy as np

from oracle import oracle as orc
from tests.qpp_helpers import gaussian_ket, haar_unitary


class NumpyLocal:
    """A rank's share held in host memory; gates through the oracle (test infrastructure)."""

    def __init__(self, nl):
        self.nl = nl
        self.amps = np.zeros(1 << nl, dtype=np.complex128)

    def view(self):
        import torch
        return torch.from_numpy(self.amps.view(np.float64))

    def sync(self):
        pass

    def apply(self, U, targets):
        self.amps[:] = orc.apply(self.amps, U, targets, [2] * self.nl)

    def apply_ctrl(self, U, ctrl, targets):
        self.amps[:] = orc.applyCTRL(self.amps, U, ctrl, targets, [2] * self.nl)

    def norm2(self):
        return float(np.vdot(self.amps, self.amps).real)

    def scale(self, s):
        self.amps *= s

    def upload(self, a):
        self.amps[:] = a

    def numpy(self):
        return self.amps.copy()


def random_program(n, seed, length=40):
    """(kind, U, ctrl, targets) steps touching every qubit, global ones included."""
    rng = np.random.default_rng(seed)
    prog = []
    for i in range(length):
        r = rng.random()
        if r < 0.45:
            t = [int(rng.integers(n))]
            prog.append(("gate", haar_unitary(rng, 2), [], t))
        elif r < 0.8:
            t = [int(x) for x in rng.choice(n, 2, replace=False)]
            prog.append(("gate", haar_unitary(rng, 4), [], t))
        else:
            q = [int(x) for x in rng.choice(n, 3, replace=False)]
            nc = 1 + int(rng.integers(2))
            prog.append(("ctrl", haar_unitary(rng, 2), q[:nc], [q[nc]]))
    return prog


def oracle_run(psi, n, prog):
    dims = [2] * n
    for kind, U, ctrl, t in prog:
        psi = orc.apply(psi, U, t, dims) if kind == "gate" else orc.applyCTRL(psi, U, ctrl, t, dims)
    return psi


def run_program(dk, prog):
    for kind, U, ctrl, t in prog:
        if kind == "gate":
            dk.apply(U, t)
        else:
            dk.apply_ctrl(U, ctrl, t)


def start_ket(n, seed):
    return gaussian_ket(np.random.default_rng(seed), 1 << n)
