"""Shared-memory trajectory kernel (one CTA per noisy shot).

Each shot's final state (dumped), its measurement outcomes and its noise
events are replayed through the oracle with qpp's QNoisyEngine semantics
(qnoisy_engine.hpp:105-121: before every step each non-measured qubit
suffers the picked Pauli; measure_seq for Z measurements) and must agree
within the complex64 tolerance (2e-5 relative, max-norm). Final samples
follow the Born rule (chi-square).
"""
import ctypes as ct

import numpy as np
import pytest

from oracle import oracle as orc
from tests.qpp_helpers import X, Y, Z, haar_unitary

pytestmark = pytest.mark.gpu
PAULI = {1: X, 2: Y, 3: Z}


def run_traj(qb, ctx, circ, nq, p, shots, seed, max_events=64):
    L = qb.lib()
    nc = max(circ.nc, 1)
    samples = np.zeros(shots, dtype=np.uint64)
    dits = np.zeros(shots * nc, dtype=np.uint32)
    dump = np.zeros(shots * 2 * 2 ** nq, dtype=np.float64)
    ev = np.zeros(shots * max_events * 2, dtype=np.uint32)
    qb.check(L.qgpu_trajectories(ctx.h, circ.h, ct.c_double(p), ct.c_uint64(shots),
                                 ct.c_uint64(seed), samples.ctypes.data_as(ct.c_void_p),
                                 dits.ctypes.data_as(ct.c_void_p), dump.ctypes.data_as(ct.c_void_p),
                                 ev.ctypes.data_as(ct.c_void_p), ct.c_uint32(max_events)))
    states = dump.reshape(shots, 2 ** nq, 2)
    states = states[..., 0] + 1j * states[..., 1]
    return samples, dits.reshape(shots, nc), states, ev.reshape(shots, max_events, 2)


def random_program(rng, nq, nsteps, measure=True, destructive=False):
    steps, creg, alive = [], 0, list(range(nq))
    for _ in range(nsteps):
        r = rng.random()
        if measure and r < 0.12 and len(alive) > 3:
            q = int(rng.choice(alive))
            steps.append(("measure", [q], creg, destructive))
            creg += 1
            if destructive:
                alive.remove(q)
        elif r < 0.3:
            sub = [int(x) for x in rng.choice(alive, size=3, replace=False)]
            steps.append(("ctrl", haar_unitary(rng, 2), sub[:2], sub[2:]))
        elif r < 0.65:
            steps.append(("gate", haar_unitary(rng, 2), [int(rng.choice(alive))]))
        else:
            t = [int(x) for x in rng.choice(alive, size=2, replace=False)]
            steps.append(("gate", haar_unitary(rng, 4), t))
    return steps, creg


def build(qb, steps, nq, nc):
    c = qb.Circuit(nq, 2, max(nc, 1))
    for st in steps:
        if st[0] == "gate":
            c.gate(st[1], st[2])
        elif st[0] == "ctrl":
            c.CTRL(st[1], st[2], st[3])
        else:
            c.measure(st[1], st[2], destructive=st[3])
    return c


def replay(steps, nq, outcomes, events):
    """Oracle replay of one shot; instruction index == step index here
    (every step compiles to one instruction)."""
    psi = np.zeros(2 ** nq, dtype=np.complex128)
    psi[0] = 1
    dims = [2] * nq
    measured = [False] * nq
    by_ins = {}
    for ins, w in events:
        if ins == 0xffffffff:
            continue
        by_ins.setdefault(int(ins), []).append((int(w) & 0xffff, int(w) >> 16))

    def rel(q):
        return sum(1 for i in range(q) if not measured[i])

    for k, st in enumerate(steps):
        for bit, pk in sorted(by_ins.get(k, [])):
            q = nq - 1 - bit
            psi = orc.apply(psi, PAULI[pk], [rel(q)], dims)
        if st[0] == "gate":
            psi = orc.apply(psi, st[1], [rel(q) for q in st[2]], dims)
        elif st[0] == "ctrl":
            psi = orc.applyCTRL(psi, st[1], [rel(q) for q in st[2]], [rel(q) for q in st[3]], dims)
        else:
            _, t, creg, destr = st
            _, _, psi, dims = orc.measure_seq(psi, [rel(t[0])], dims, destr,
                                              forced=[int(outcomes[creg])])
            if destr:
                measured[t[0]] = True
    return psi, measured


def fixed_part(state, nq, measured, outcomes_by_qubit):
    """Amplitudes of a full register whose measured qubits sit at their
    outcomes, in the order of the remaining qubits."""
    idx = []
    for i in range(2 ** nq):
        ok = all(((i >> (nq - 1 - q)) & 1) == outcomes_by_qubit[q]
                 for q in range(nq) if measured[q])
        if ok:
            idx.append(i)
    return state[idx]


@pytest.mark.parametrize("p,destructive", [(0.0, False), (0.03, False), (0.03, True)])
def test_shots_replay_through_oracle(ctx, p, destructive):
    import qpp_b200 as qb
    rng = np.random.default_rng(int(p * 1000) + destructive)
    nq = 9
    steps, nc = random_program(rng, nq, 50, destructive=destructive)
    c = build(qb, steps, nq, nc)
    shots = 24
    samples, dits, states, events = run_traj(qb, ctx, c, nq, p, shots, seed=99)
    n_err = 0
    for s in range(shots):
        ref, measured = replay(steps, nq, dits[s], events[s])
        outq = {}
        for st in steps:
            if st[0] == "measure":
                outq[st[1][0]] = int(dits[s][st[2]])
        got = fixed_part(states[s], nq, measured, outq) if destructive else states[s]
        assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) < 2e-5
        n_err += int(np.sum(events[s][:, 0] != 0xffffffff))
    if p > 0:
        assert n_err > 0


def test_final_samples_follow_born_rule(ctx):
    import qpp_b200 as qb
    rng = np.random.default_rng(8)
    nq = 3
    c = qb.Circuit(nq, 2, 1)
    c.gate(haar_unitary(rng, 4), [0, 1]).gate(haar_unitary(rng, 4), [1, 2])
    c.gate(haar_unitary(rng, 2), [0])
    shots = 20000
    samples, _, states, _ = run_traj(qb, ctx, c, nq, 0.0, shots, seed=5)
    probs = np.abs(states[0]) ** 2
    counts = np.bincount(samples.astype(np.int64), minlength=8)
    chi2 = float(np.sum((counts - shots * probs) ** 2 / np.maximum(shots * probs, 1e-12)))
    assert chi2 < 24.3  # 7 dof, p = 0.001


def test_tiled_registers_match_untiled_and_oracle(ctx):
    """16-qubit registers run in a global slot; the tile passes (widths 9 and
    12) must give bit-identical shots, samples, outcomes and noise events to
    the untiled form, including passes split by noise, and agree with the
    oracle replay."""
    import qpp_b200 as qb
    rng = np.random.default_rng(16)
    nq = 16
    steps, nc = random_program(rng, nq, 36, destructive=False)
    c = build(qb, steps, nq, nc)
    shots, p = 4, 0.02
    runs = {}
    try:
        for T in (0, 9, 12):
            assert qb.traj_tile_width(ctx, nq, T) == T
            runs[T] = run_traj(qb, ctx, c, nq, p, shots, seed=7)
    finally:
        qb.traj_tile_width(ctx, nq, -2)
    for T in (9, 12):
        for a, b in zip(runs[0], runs[T]):
            assert np.array_equal(a, b), T
    samples, dits, states, events = runs[0]
    assert int(np.sum(events[:, :, 0] != 0xffffffff)) > 0
    for s in range(2):
        ref, _ = replay(steps, nq, dits[s], events[s])
        assert np.max(np.abs(states[s] - ref)) / np.max(np.abs(ref)) < 2e-5
