"""Device engines: QEngine / QDensityEngine / QNoisyEngine semantics.

* teleportation (the reference's unit_tests/tests/qasm/qasm.cpp:82-94 on
  unit_tests/tests/qasm/circuits/units/teleportation.qasm, restated as
  circuit steps): the teleported qubit ends in |0> for every outcome;
* replay parity: the engine's recorded outcomes and Kraus picks, replayed
  through an oracle-driven engine loop (qengine.hpp / qnoisy_engine.hpp
  semantics: noise on every non-measured qudit before every step, relative
  positions after destructive measurements), give the same final state,
  dits and probabilities within 1e-12;
* free-running parity: with the same mt19937 seed the engine draws the same
  measurement outcome as the oracle's measure_seq (std::discrete_distribution
  over the full basis);
* outcome statistics follow the Born rule.
"""
import numpy as np
import pytest

from oracle import oracle as orc
from tests.qpp_helpers import (CNOT, H, X, Z, amplitude_damping_kraus, depolarizing_kraus,
                               gaussian_ket, haar_unitary, prj)

pytestmark = pytest.mark.gpu


def u3(theta, phi, lam):
    c, s = np.cos(theta / 2), np.sin(theta / 2)
    return np.array([[c, -np.exp(1j * lam) * s],
                     [np.exp(1j * phi) * s, np.exp(1j * (phi + lam)) * c]], dtype=np.complex128)


def teleport_circuit(qb):
    c = qb.Circuit(3, 2, 2)
    c.gate(H, [1]).gate(CNOT, [1, 2])               # Bell pair on b[0], b[1]
    c.gate(u3(0.3, 0.2, 0.1), [0])                  # state to teleport on a[0]
    c.gate(CNOT, [0, 1]).gate(H, [0])
    c.measure([0], 0, destructive=False)            # a[0] -> c
    c.measure([1], 1, destructive=False)            # b[0] -> d
    c.cCTRL(X, [1], [2])                            # if (d == 1) x b[1]
    c.cCTRL(Z, [0], [2])                            # if (c == 1) z b[1]
    c.gate(u3(-0.3, -0.1, -0.2), [2])               # u3^dagger
    return c


@pytest.mark.parametrize("kind", ["ket", "rho"])
def test_teleportation(ctx, kind):
    import qpp_b200 as qb
    c = teleport_circuit(qb)
    seen = set()
    for seed in range(12):
        e = qb.Engine(ctx, c, qb.KET if kind == "ket" else qb.RHO).set_seed(seed).execute()
        st = e.get_state()
        rho = orc.ptrace(st.numpy(), [0, 1], [2, 2, 2])
        assert np.linalg.norm(rho - prj(np.array([1, 0]))) < 1e-5
        seen.add(tuple(e.get_dits()[0]))
    assert len(seen) > 1  # different outcomes, same teleported state


# ----------------------------------------------------- oracle engine loop
def oracle_engine(steps, nq, nc, psi0, outcomes, noise, Ks=None):
    """qengine.hpp / qnoisy_engine.hpp restated over the oracle functions,
    with every random choice forced from the recorded lists."""
    state = psi0.copy()
    dims = [2] * nq
    measured = [False] * nq
    dits, probs = [0] * nc, [0.0] * nc
    oi, ni = 0, 0

    def rel(q):
        return sum(1 for i in range(q) if not measured[i])

    for st in steps:
        if Ks is not None:
            for q in range(nq):
                if measured[q]:
                    continue
                k = noise[ni]
                ni += 1
                state = orc.apply(state, Ks[k], [rel(q)], dims)
                state = orc.normalize(state)
        kind = st[0]
        if kind == "gate":
            _, U, t = st
            state = orc.apply(state, U, [rel(q) for q in t], dims)
        elif kind == "ctrl":
            _, U, cl, t = st
            state = orc.applyCTRL(state, U, [rel(q) for q in cl], [rel(q) for q in t], dims)
        elif kind == "measure":
            _, t, creg, destr = st
            forced = outcomes[oi:oi + len(t)]
            oi += len(t)
            res, ps, state, dims = orc.measure_seq(state, [rel(q) for q in t], dims, destr,
                                                   forced=forced)
            for i, (r, p) in enumerate(zip(res, ps)):
                dits[creg + i], probs[creg + i] = r, p
            if destr:
                for q in t:
                    measured[q] = True
    return state, dits, probs


def random_steps(rng, nq, nsteps, with_measure=True):
    steps, creg = [], 0
    alive = list(range(nq))
    for i in range(nsteps):
        r = rng.random()
        if with_measure and r < 0.15 and len(alive) > 4:
            k = 1 + int(rng.integers(2))  # leaves >= 3 alive for 3-qubit steps
            t = [int(x) for x in rng.choice(alive, size=k, replace=False)]
            destr = bool(rng.random() < 0.5)
            steps.append(("measure", t, creg, destr))
            creg += k
            if destr:
                alive = [q for q in alive if q not in t]
        elif r < 0.35 and len(alive) >= 3:
            sub = [int(x) for x in rng.choice(alive, size=3, replace=False)]
            steps.append(("ctrl", haar_unitary(rng, 2), sub[:2], sub[2:]))
        else:
            k = 1 + int(rng.integers(2))
            t = [int(x) for x in rng.choice(alive, size=k, replace=False)]
            steps.append(("gate", haar_unitary(rng, 2 ** k), t))
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


@pytest.mark.parametrize("noise", [None, "depolarizing", "amplitude_damping"])
def test_replay_parity_with_oracle_engine(ctx, noise):
    import qpp_b200 as qb
    rng = np.random.default_rng({None: 1, "depolarizing": 2, "amplitude_damping": 3}[noise])
    nq = 8
    steps, nc = random_steps(rng, nq, 40)
    c = build(qb, steps, nq, nc)
    psi0 = gaussian_ket(rng, 2 ** nq)
    e = qb.Engine(ctx, c).set_seed(17).set_state(qb.State.from_numpy(ctx, psi0, [2] * nq))
    Ks = None
    if noise == "depolarizing":
        Ks = depolarizing_kraus(0.05)
        e.set_noise(Ks, [0.95, 0.05 / 3, 0.05 / 3, 0.05 / 3])
    elif noise == "amplitude_damping":
        Ks = amplitude_damping_kraus(0.1)
        e.set_noise(Ks)  # state-dependent
    e.execute()
    outcomes, picks = e.get_record()
    got = e.get_state().numpy()
    dits, probs = e.get_dits()
    ref, rdits, rprobs = oracle_engine(steps, nq, max(nc, 1), psi0, outcomes, picks, Ks)
    assert got.shape == ref.shape
    assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) < 1e-12
    assert dits == rdits[:len(dits)]
    assert np.allclose(probs, rprobs[:len(probs)], rtol=1e-12, atol=1e-14)
    if noise == "depolarizing":
        assert any(k != 0 for k in picks)  # some non-identity Kraus picked


def test_free_running_outcome_matches_oracle_rng(ctx):
    """Same std::mt19937 seed -> same full-basis draw as qpp's sample()."""
    import qpp_b200 as qb
    rng = np.random.default_rng(5)
    nq = 10
    agree = 0
    for seed in range(20):
        psi = gaussian_ket(rng, 2 ** nq)
        c = qb.Circuit(nq, 2, 3).measure([2, 7, 4], 0, destructive=False)
        e = qb.Engine(ctx, c).set_seed(seed).set_state(qb.State.from_numpy(ctx, psi, [2] * nq))
        dits, _ = e.execute().get_dits()
        res, _, _, _ = orc.measure_seq(psi, [2, 7, 4], [2] * nq, False, seed=seed)
        agree += dits == res
    assert agree == 20


def test_measurement_statistics_follow_born_rule(ctx):
    import qpp_b200 as qb
    psi = np.array([np.sqrt(0.1), np.sqrt(0.2), np.sqrt(0.3), np.sqrt(0.4)], dtype=np.complex128)
    c = qb.Circuit(2, 2, 2).measure([0, 1], 0)
    e = qb.Engine(ctx, c).set_seed(3).set_state(qb.State.from_numpy(ctx, psi, [2, 2]))
    n = 4000
    stats = e.execute(n).get_stats()
    expect = {(0, 0): 0.1, (0, 1): 0.2, (1, 0): 0.3, (1, 1): 0.4}
    chi2 = sum((stats.get(k, 0) - n * p) ** 2 / (n * p) for k, p in expect.items())
    assert sum(stats.values()) == n
    assert chi2 < 16.3  # 3 dof, p = 0.001
