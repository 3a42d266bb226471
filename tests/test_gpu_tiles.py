"""Plain form of qgpu_run_gates on qubit kets: runs of 1- and 2-qubit gates
(plain, fan, controlled, shifted controls) as tile passes in shared memory.

Parity: complex128 within 1e-12 relative (max-norm) of the oracle applying
qpp's gates one by one; against the library's own one-launch-per-gate path
(State.apply / apply_ctrl) within 1e-14 (the same arithmetic per amplitude;
only the compiler's contraction of the two paths may differ); complex64
within 1e-5 of the oracle. Tile sizes 5..14 bits and states from 3 to 20
qubits, so single-tile states, tiles smaller than the state and every low-bit
layout are covered."""
import ctypes as ct

import numpy as np
import pytest

from oracle import oracle as orc
from tests.qpp_helpers import gaussian_ket, haar_unitary

pytestmark = pytest.mark.gpu


def relerr(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def _random_steps(rng, n, count):
    steps = []
    for _ in range(count):
        r = rng.random()
        perm = [int(x) for x in rng.permutation(n)]
        if r < 0.45 or n < 3:
            steps.append(("gate", haar_unitary(rng, 2), [perm[0]]))
        elif r < 0.7:
            steps.append(("gate", haar_unitary(rng, 4), perm[:2]))
        elif r < 0.8:
            k = int(rng.integers(1, 4))
            steps.append(("fan", haar_unitary(rng, 2), perm[:k]))
        else:
            nc = int(rng.integers(1, min(3, n - 2) + 1))
            nt = 2 if rng.random() < 0.3 else 1
            shift = [int(x) for x in rng.integers(0, 2, size=nc)] if rng.random() < 0.4 else None
            steps.append(("ctrl", haar_unitary(rng, 2 ** nt), perm[:nc], perm[nc:nc + nt], shift))
    return steps


def _circuit(qb, n, steps):
    c = qb.Circuit(n)
    for st in steps:
        if st[0] == "gate":
            c.gate(st[1], st[2])
        elif st[0] == "fan":
            c.gate_fan(st[1], st[2])
        else:
            c.CTRL(st[1], st[2], st[3], shift=st[4])
    return c


def _oracle(psi, n, steps):
    dims = [2] * n
    for st in steps:
        if st[0] == "gate":
            psi = orc.apply(psi, st[1], st[2], dims)
        elif st[0] == "fan":
            for t in st[2]:
                psi = orc.apply(psi, st[1], [t], dims)
        else:
            psi = orc.applyCTRL(psi, st[1], st[2], st[3], dims, shift=st[4])
    return psi


def _per_gate(s, steps):
    for st in steps:
        if st[0] == "gate":
            s.apply(st[1], st[2])
        elif st[0] == "fan":
            for t in st[2]:
                s.apply(st[1], [t])
        else:
            s.apply_ctrl(st[1], st[2], st[3], shift=st[4])
    return s


@pytest.mark.parametrize("n,bits", [(3, 0), (9, 0), (12, 0), (14, 0), (14, 5), (14, 8),
                                    (16, 12), (16, 14), (18, 0), (20, 11)])
def test_tile_passes_match_oracle_and_per_gate(ctx, n, bits):
    import qpp_b200 as qb
    rng = np.random.default_rng(100 + n + bits)
    steps = _random_steps(rng, n, 80)
    psi = gaussian_ket(rng, 2 ** n)
    ref = _oracle(psi.copy(), n, steps)
    qb.check(qb.lib().qgpu_ctx_set_tile_bits(ctx.h, ct.c_int(bits)))
    try:
        s = qb.State.from_numpy(ctx, psi, [2] * n)
        _circuit(qb, n, steps).run(s, qb.PLAIN)
        got = s.numpy()
    finally:
        qb.check(qb.lib().qgpu_ctx_set_tile_bits(ctx.h, ct.c_int(0)))
    assert relerr(got, ref) < 1e-12
    one = _per_gate(qb.State.from_numpy(ctx, psi, [2] * n), steps).numpy()
    assert relerr(got, one) < 1e-14


@pytest.mark.parametrize("n", [10, 15])
def test_tile_passes_complex64(ctx, n):
    import qpp_b200 as qb
    rng = np.random.default_rng(200 + n)
    steps = _random_steps(rng, n, 60)
    psi = gaussian_ket(rng, 2 ** n).astype(np.complex64).astype(np.complex128)
    ref = _oracle(psi.copy(), n, steps)
    s = qb.State.from_numpy(ctx, psi, [2] * n, qb.C64)
    _circuit(qb, n, steps).run(s, qb.PLAIN)
    assert relerr(s.numpy(), ref) < 1e-5


def test_config1_through_run_gates(ctx):
    """The 20-qubit sequence of the gate benchmark (1000 Haar gates, 70% 1q /
    30% 2q, then 100 applyCTRL with 1-3 controls) as one qgpu_run_gates call
    in the plain form, against the oracle within 1e-12."""
    import qpp_b200 as qb
    from qpp_b200.workloads import ket_gate_sequence
    n = 20
    seq = ket_gate_sequence(n, seed=3)
    rng = np.random.default_rng(3)
    psi = gaussian_ket(rng, 2 ** n)
    c = qb.Circuit(n)
    for U, cs, t in seq:
        c.CTRL(U, cs, t) if cs else c.gate(U, t)
    s = qb.State.from_numpy(ctx, psi, [2] * n)
    c.run(s, qb.PLAIN)
    ref = psi.copy()
    for U, cs, t in seq:
        ref = orc.applyCTRL(ref, U, cs, t, [2] * n, path=1) if cs else \
            orc.apply(ref, U, t, [2] * n, path=1)
    assert relerr(s.numpy(), ref) < 1e-12


def test_tile_bits_range(ctx):
    import qpp_b200 as qb
    L = qb.lib()
    for bad in (4, 15, -1):
        with pytest.raises(qb.OutOfRange):
            qb.check(L.qgpu_ctx_set_tile_bits(ctx.h, ct.c_int(bad)))
    qb.check(L.qgpu_ctx_set_tile_bits(ctx.h, ct.c_int(0)))
