"""Batched uneven instances: one CUDA-graph launch versus the plain loop.

Kets of 10-16 qubits and density matrices of 4-9 qubits, each with its own
random layered circuit (density matrices: a depolarising channel p=0.005 on
every qubit after each layer, and every other one a 16-operator channel on a
pair), complex64. Registers above 2^14 amplitudes (kets of 15-16 qubits,
density matrices of 8-9 qubits) run in place in their own states. The graph form must agree with the
plain per-instance loop on the same inputs within 2e-5 relative (max-norm),
and a sample of instances with the complex128 oracle within 1e-4.
"""
import numpy as np
import pytest

from oracle import oracle as orc
from tests.qpp_helpers import depolarizing_kraus, gaussian_ket, haar_unitary, random_rho

pytestmark = pytest.mark.gpu


def layered(qb, rng, n, depth, rho, pair=False):
    c = qb.Circuit(n)
    steps = []
    for _ in range(depth):
        for q in range(n):
            U = haar_unitary(rng, 2)
            c.gate(U, [q])
            steps.append(("g", U, [q]))
        perm = rng.permutation(n)
        for i in range(n // 2):
            U = haar_unitary(rng, 4)
            t = [int(perm[2 * i]), int(perm[2 * i + 1])]
            c.gate(U, t)
            steps.append(("g", U, t))
        if rho:
            for q in range(n):
                from qpp_b200.serving import c_channel
                c_channel(c, depolarizing_kraus(0.005), [q])
                steps.append(("k", depolarizing_kraus(0.005), [q]))
            if pair:
                from qpp_b200.serving import c_channel, pair_channel
                t = [int(x) for x in rng.choice(n, 2, replace=False)]
                c_channel(c, pair_channel(), t)
                steps.append(("k", pair_channel(), t))
    return c, steps


def test_graph_batch_matches_plain_loop_and_oracle(ctx):
    import qpp_b200 as qb
    rng = np.random.default_rng(2048)
    circuits, inputs, kinds, all_steps = [], [], [], []
    for i in range(40):
        rho = i % 5 == 4
        n = int(rng.integers(4, 10)) if rho else int(rng.integers(10, 17))
        c, steps = layered(qb, rng, n, 3, rho, pair=rho and i % 10 == 9)
        circuits.append(c)
        all_steps.append(steps)
        kinds.append(qb.RHO if rho else qb.KET)
        inputs.append(random_rho(rng, 2 ** n, 8) if rho else gaussian_ket(rng, 2 ** n))
    a = [qb.State.from_numpy(ctx, x, [2] * int(np.log2(len(x))), qb.C64) for x in inputs]
    b = [qb.State.from_numpy(ctx, x, [2] * int(np.log2(len(x))), qb.C64) for x in inputs]
    kernels = qb.run_batch(ctx, circuits, a, qb.FUSED)
    qb.run_batch(ctx, circuits, b, qb.PLAIN)
    assert kernels >= 2  # several register sizes in one graph
    for i in range(len(circuits)):
        ga, gb = a[i].numpy(), b[i].numpy()
        assert np.max(np.abs(ga - gb)) / np.max(np.abs(gb)) < 2e-5, i
    big = [i for i in range(len(circuits)) if kinds[i] == qb.RHO and inputs[i].shape[0] >= 256]
    assert big, "no in-place density matrix in the sample"
    for i in sorted({0, 4, 9, 14, big[0]}):
        x = inputs[i]
        n = int(round(np.log2(x.shape[0])))
        dims = [2] * n
        for kind, M, t in all_steps[i]:
            x = orc.apply(x, M, t, dims) if kind == "g" else orc.apply_kraus(x, M, t, dims)
        got = a[i].numpy()
        assert np.max(np.abs(got - x)) / np.max(np.abs(x)) < 1e-4, i


def test_batch_rejects_a_state_given_twice(ctx):
    import qpp_b200 as qb
    c = qb.Circuit(3)
    c.gate(np.eye(2), [0])
    s = qb.State(ctx, qb.KET, [2] * 3, qb.C64)
    with pytest.raises(qb.Duplicates):
        qb.run_batch(ctx, [c, c], [s, s], qb.FUSED)
    s.free()


@pytest.mark.parametrize("w", [2, 3, 4])
def test_every_fusion_width_matches_plain_loop(ctx, w):
    """Pinned fusion widths 2-4 (8 x 8 and 16 x 16 blocks) on kets of 10-16
    qubits and density matrices of 4-9: the graph form agrees with the plain
    per-instance loop within 2e-5 relative."""
    import qpp_b200 as qb
    rng = np.random.default_rng(77 + w)
    circuits, inputs = [], []
    for i in range(16):
        rho = i % 4 == 3
        n = int(rng.integers(4, 10)) if rho else int(rng.integers(10, 17))
        c, _ = layered(qb, rng, n, 3, rho)
        circuits.append(c)
        inputs.append(random_rho(rng, 2 ** n, 8) if rho else gaussian_ket(rng, 2 ** n))
    sizes = sorted({int(np.log2(x.shape[0])) * (2 if x.ndim == 2 else 1) for x in inputs})
    try:
        for n in sizes:
            assert qb.traj_fusion_width(ctx, n, w) == w
        a = [qb.State.from_numpy(ctx, x, [2] * int(np.log2(len(x))), qb.C64) for x in inputs]
        b = [qb.State.from_numpy(ctx, x, [2] * int(np.log2(len(x))), qb.C64) for x in inputs]
        qb.run_batch(ctx, circuits, a, qb.FUSED)
        qb.run_batch(ctx, circuits, b, qb.PLAIN)
        for i in range(len(circuits)):
            ga, gb = a[i].numpy(), b[i].numpy()
            assert np.max(np.abs(ga - gb)) / np.max(np.abs(gb)) < 2e-5, (w, i)
    finally:
        for n in sizes:
            qb.traj_fusion_width(ctx, n, -2)


def test_block_layered_registers_match_plain_loop(ctx):
    """Kets of 20-21 qubits and density matrices of 10 and 12 qubits (20 and
    24 virtual qubits) run block-layered (programs fused into blocks of <= 4
    (virtual) qubits, launch j applying block j of every such register),
    beside a 16-qubit ket on the layered tile passes and small instances in
    shared memory, and agree with the plain per-instance loop within 2e-5
    relative."""
    import qpp_b200 as qb
    rng = np.random.default_rng(2020)
    spec = [("k", 20), ("k", 21), ("k", 16), ("k", 11), ("r", 10), ("r", 12), ("r", 8), ("r", 5)]
    circuits, inputs = [], []
    for kind, n in spec:
        c, _ = layered(qb, rng, n, 2, kind == "r", pair=kind == "r")
        circuits.append(c)
        inputs.append(random_rho(rng, 2 ** n, 4) if kind == "r" else gaussian_ket(rng, 2 ** n))
    a = [qb.State.from_numpy(ctx, x, [2] * int(np.log2(len(x))), qb.C64) for x in inputs]
    b = [qb.State.from_numpy(ctx, x, [2] * int(np.log2(len(x))), qb.C64) for x in inputs]
    kernels = qb.run_batch(ctx, circuits, a, qb.FUSED)
    assert qb.batch_last_phases(ctx)["plain_ms"] < 50  # nothing fell back to the loop
    qb.run_batch(ctx, circuits, b, qb.PLAIN)
    assert kernels > 20  # the branch passes are graph kernels too
    for i in range(len(circuits)):
        ga, gb = a[i].numpy(), b[i].numpy()
        assert np.max(np.abs(ga - gb)) / np.max(np.abs(gb)) < 2e-5, spec[i]
    for s in a + b:
        s.free()
