"""Fused complex64 form: 6-qubit tcgen05 blocks with split-FP16 products.

Tolerances: a single block agrees with the complex128 oracle within 1e-5
relative (max-norm) -- FP32 accumulation of 3 x FP16 split products of
power-of-two-scaled operands; the identity block reproduces its input within
2^-20 relative (hi and lo keep 11 significant bits each); a fused layered
circuit keeps fidelity >= 1 - 1e-6 against the plain complex128 form.
A bounded wait that runs out reports QGPU_ERR_TIMEOUT and leaves the
context usable.
"""
import ctypes as ct

import numpy as np
import pytest

from oracle import oracle as orc
from tests.qpp_helpers import gaussian_ket, haar_unitary

pytestmark = pytest.mark.gpu


def relerr(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def test_identity_block_reproduces_input(ctx):
    import qpp_b200 as qb
    rng = np.random.default_rng(1)
    n = 14
    psi = gaussian_ket(rng, 2 ** n).astype(np.complex64).astype(np.complex128)
    s = qb.State.from_numpy(ctx, psi, [2] * n, qb.C64)
    qb.apply_tc(s, np.eye(64), [0, 3, 5, 8, 11, 13])
    got = s.numpy()
    assert np.max(np.abs(got - psi) / np.maximum(np.abs(psi), 1e-30)) < 2 ** -20


@pytest.mark.parametrize("n,targets", [(13, [0, 1, 2, 3, 4, 5]), (14, [13, 12, 11, 10, 9, 8]),
                                       (15, [2, 9, 0, 14, 7, 4]), (16, [5, 1, 11]),
                                       (16, [15]), (18, [3, 17, 8, 0, 12, 6])])
def test_block_matches_oracle(ctx, n, targets):
    import qpp_b200 as qb
    rng = np.random.default_rng(n + len(targets))
    psi = gaussian_ket(rng, 2 ** n).astype(np.complex64).astype(np.complex128)
    U = haar_unitary(rng, 2 ** len(targets))
    s = qb.State.from_numpy(ctx, psi, [2] * n, qb.C64)
    qb.apply_tc(s, U, targets)
    ref = orc.apply(psi, U, targets, [2] * n)
    assert relerr(s.numpy(), ref) < 1e-5


def test_fused_layered_circuit_fidelity(ctx):
    import qpp_b200 as qb
    n, depth = 18, 10
    c = qb.layered_circuit(n, depth, 7)
    p128 = qb.State(ctx, qb.KET, [2] * n, qb.C128).fill_gaussian(5)
    p64 = qb.State(ctx, qb.KET, [2] * n, qb.C64).convert_from(p128)
    c.run(p128, qb.PLAIN)
    c.run(p64, qb.FUSED)
    a, b = p128.numpy(), p64.numpy()
    fid = abs(np.vdot(a, b)) ** 2 / (np.vdot(a, a).real * np.vdot(b, b).real)
    assert 1 - fid < 1e-6, 1 - fid
    # and the plain complex128 run itself matches the oracle gate by gate
    psi = qb.State(ctx, qb.KET, [2] * n, qb.C128).fill_gaussian(5).numpy()
    from qpp_b200 import workloads
    for layer in workloads.layered_circuit(n, depth, 7):
        for U, t in layer:
            psi = orc.apply(psi, U, t, [2] * n, path=1)
    assert relerr(a, psi) < 1e-12


@pytest.mark.parametrize("n,n_gates", [(9, 120), (20, 300), (23, 60)])
def test_fused_complex128_circuit_matches_oracle(ctx, n, n_gates):
    """The fused form in complex128: blocks of <= 2 qubits as tile passes up
    to 22 qubits, blocks of <= 3 qubits as dense passes above. The circuit
    mixes 1- and 2-qubit gates with controlled gates of 1-3 controls (some
    with shifts) in between, a fan gate and a 3-qubit gate (steps the
    planner leaves unfused); within 1e-12 of the oracle applying the steps one
    by one."""
    import qpp_b200 as qb
    from qpp_b200.workloads import ket_gate_sequence
    rng = np.random.default_rng(n)
    seq = ket_gate_sequence(n, seed=n, n_gates=n_gates, n_ctrl=n_gates // 10)
    plain, ctrl = seq[:n_gates], seq[n_gates:]
    steps = []  # (kind, U, ctrl, target, shift)
    for i, (U, c, t) in enumerate(plain):
        steps.append(("gate", U, c, t, None))
        if i % 10 == 5 and ctrl:
            U2, c2, t2 = ctrl.pop()
            shift = [int(x) for x in rng.integers(0, 2, size=len(c2))] if i % 20 == 5 else None
            steps.append(("ctrl", U2, c2, t2, shift))
        if i == n_gates // 2:
            steps.append(("fan", haar_unitary(rng, 2), [], [0, n - 1, n // 2], None))
            steps.append(("gate", haar_unitary(rng, 8), [], [1, n - 2, n // 3], None))
    c = qb.Circuit(n)
    for kind, U, cs, t, sh in steps:
        if kind == "gate":
            c.gate(U, t)
        elif kind == "fan":
            c.gate_fan(U, t)
        else:
            c.CTRL(U, cs, t, shift=sh)
    s = qb.State(ctx, qb.KET, [2] * n, qb.C128).fill_gaussian(3)
    psi = s.numpy()
    c.run(s, qb.FUSED)
    dims = [2] * n
    for kind, U, cs, t, sh in steps:
        if kind == "gate":
            psi = orc.apply(psi, U, t, dims)
        elif kind == "fan":
            for q in t:
                psi = orc.apply(psi, U, [q], dims)
        else:
            psi = orc.applyCTRL(psi, U, cs, t, dims, shift=sh)
    assert relerr(s.numpy(), psi) < 1e-12


@pytest.mark.parametrize("scale", [1.0, 2.0 ** -40, 2.0 ** 30])
def test_block_scale_follows_the_norm(ctx, scale):
    """The fp16 scale comes from |psi|: unnormalised kets keep the accuracy."""
    import qpp_b200 as qb
    rng = np.random.default_rng(11)
    n = 15
    psi = (gaussian_ket(rng, 2 ** n) * scale).astype(np.complex64).astype(np.complex128)
    U = haar_unitary(rng, 64)
    targets = [14, 1, 7, 3, 10, 0]
    s = qb.State.from_numpy(ctx, psi, [2] * n, qb.C64)
    qb.apply_tc(s, U, targets)
    ref = orc.apply(psi, U, targets, [2] * n)
    assert relerr(s.numpy(), ref) < 1e-5


def test_wait_runs_out_then_context_recovers(ctx):
    """The next fused pass first waits on a barrier that nothing completes:
    the wait gives up after its iteration limit, the call reports Timeout,
    and the same context then runs a pass that matches the oracle."""
    import qpp_b200 as qb
    rng = np.random.default_rng(12)
    n = 14
    targets = [0, 2, 4, 6, 8, 10]
    psi = gaussian_ket(rng, 2 ** n).astype(np.complex64).astype(np.complex128)
    U = haar_unitary(rng, 64)
    L = qb.lib()
    s = qb.State.from_numpy(ctx, psi, [2] * n, qb.C64)
    qb.check(L.qgpu_ctx_set_wait_test(ctx.h, ct.c_uint32(4096), ct.c_int(1)))
    try:
        with pytest.raises(qb.Timeout):
            qb.apply_tc(s, U, targets)
    finally:
        qb.check(L.qgpu_ctx_set_wait_test(ctx.h, ct.c_uint32(0), ct.c_int(0)))
    s2 = qb.State.from_numpy(ctx, psi, [2] * n, qb.C64)
    qb.apply_tc(s2, U, targets)
    assert relerr(s2.numpy(), orc.apply(psi, U, targets, [2] * n)) < 1e-5
