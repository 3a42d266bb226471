"""Fused superoperator form of a complex64 density matrix (Circuit.run with
FUSED on a RHO state; no reference counterpart): gates and 1- or 2-qubit
channels become superoperators on the 2n virtual qubits, merged into blocks
of at most 4 virtual qubits, one pass per block; from 11 qubits into blocks
of at most 6 virtual qubits, each a split-FP16 tcgen05 pass (checked at 12
qubits against the plain complex128 form, itself checked against the oracle). Against the FP64 oracle
(qpp's apply and Kraus apply restated) within 2e-5 relative in the max-norm
(complex64 arithmetic); against the plain complex128 form on the GPU at 12
qubits; fewer passes than the plain form; unsupported cases raise
NotSupported."""
import numpy as np
import pytest

from oracle import oracle as orc
from tests.qpp_helpers import depolarizing_kraus, haar_unitary, random_rho

pytestmark = pytest.mark.gpu

TOL = 2e-5


def relerr(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def layered_rho_circuit(qb, rng, n, depth, single=True):
    """Per layer: a Haar 1-qubit gate on every qubit, a Haar 2-qubit gate and
    the 16-operator pair channel on each pair of a random matching, and (when
    `single`) a depolarising channel on one random qubit."""
    from qpp_b200.serving import c_channel, pair_channel
    c = qb.Circuit(n)
    steps = []
    for _ in range(depth):
        for q in range(n):
            U = haar_unitary(rng, 2)
            c.gate(U, [q])
            steps.append(("g", U, [q]))
        perm = rng.permutation(n)
        for i in range(n // 2):
            t = [int(perm[2 * i]), int(perm[2 * i + 1])]
            U = haar_unitary(rng, 4)
            c.gate(U, t)
            steps.append(("g", U, t))
            c_channel(c, pair_channel(), t)
            steps.append(("k", pair_channel(), t))
        if single:
            q = int(rng.integers(n))
            c_channel(c, depolarizing_kraus(0.02), [q])
            steps.append(("k", depolarizing_kraus(0.02), [q]))
    return c, steps


@pytest.mark.parametrize("n", [1, 2, 3, 5, 6])
def test_fused_rho_matches_oracle(ctx, n):
    import qpp_b200 as qb
    rng = np.random.default_rng(300 + n)
    c, steps = layered_rho_circuit(qb, rng, n, 3)
    x = random_rho(rng, 2 ** n, 3)
    s = qb.State.from_numpy(ctx, x, [2] * n, qb.C64)
    c.run(s, qb.FUSED)
    ref = x
    dims = [2] * n
    for kind, M, t in steps:
        ref = orc.apply(ref, M, t, dims) if kind == "g" else orc.apply_kraus(ref, M, t, dims)
    assert relerr(s.numpy(), ref) < TOL


def test_fused_rho_12_qubits_against_plain_c128_and_pass_count(ctx):
    """12 qubits (a 4096 x 4096 matrix): the fused complex64 form agrees with
    the plain complex128 form within 2e-5 relative, with at most n/2 + 1
    passes per layer against the plain form's one per gate and per channel."""
    import qpp_b200 as qb
    rng = np.random.default_rng(12)
    n, depth = 12, 3
    c, steps = layered_rho_circuit(qb, rng, n, depth)
    x = random_rho(rng, 2 ** n, 8)
    a = qb.State.from_numpy(ctx, x, [2] * n, qb.C64)
    b = qb.State.from_numpy(ctx, x, [2] * n, qb.C128)
    ctx.synchronize()
    l0 = ctx.launches()
    c.run(a, qb.FUSED)
    ctx.synchronize()
    fused = ctx.launches() - l0
    l0 = ctx.launches()
    c.run(b, qb.PLAIN)
    ctx.synchronize()
    plain = ctx.launches() - l0
    assert plain == len(steps)
    assert fused <= depth * (n // 2 + 1) + 1, fused
    ga, gb = a.numpy(), b.numpy()
    assert relerr(ga, gb) < TOL
    assert abs(np.trace(ga) - np.trace(gb)) < 1e-5


def test_fused_rho_unsupported(ctx):
    import qpp_b200 as qb
    rng = np.random.default_rng(1)
    c, _ = layered_rho_circuit(qb, rng, 3, 1)
    s128 = qb.State.from_numpy(ctx, random_rho(rng, 8, 2), [2] * 3, qb.C128)
    with pytest.raises(qb.NotSupported):
        c.run(s128, qb.FUSED)
    m = qb.Circuit(3, 2, 1)
    m.gate(haar_unitary(rng, 2), [0])
    m.measure([1], 0, destructive=False)
    s64 = qb.State.from_numpy(ctx, random_rho(rng, 8, 2), [2] * 3, qb.C64)
    with pytest.raises(qb.NotSupported):
        m.run(s64, qb.FUSED)
    w = qb.Circuit(3)
    w.gate(haar_unitary(rng, 8), [0, 1, 2])
    with pytest.raises(qb.NotSupported):
        w.run(s64, qb.FUSED)
