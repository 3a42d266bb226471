"""Z-basis sampling and measurement on resident states, and the engines'
execute(reps) semantics.

* qgpu_sample draws exactly the oracle's qpp::sample draws (the same
  std::mt19937 seed, std::discrete_distribution over the full basis) for
  kets, density matrices and mixed dimensions;
* qgpu_measure_seq agrees with the oracle's measure_seq (outcomes drawn from
  the same seed, probabilities and post-measurement state within 1e-12)
  for kets and density matrices on both of qpp's paths (<= 10 and > 10
  subsystems), destructive or not, drawn or forced;
* QEngine::execute(reps) (qengine.hpp:1341-1405): the sampling form (gates,
  then only measurements) gives the oracle's draws in qpp's RNG order, also
  after the canonical reordering; otherwise the steps after the first
  measurement repeat from the same point and the engine keeps the first
  repetition; execute continues from the engine's current state; statistics
  accumulate until reset; set_state checks the size;
* qpp::measure with Kraus operators or a basis (instruments.hpp:371-712),
  reset and discard (:1148-1292) agree with the oracle: the same seeded
  outcome, probabilities and post-measurement states within 1e-12.
"""
import numpy as np
import pytest

from oracle import oracle as orc
from tests.qpp_helpers import gaussian_ket, haar_unitary, random_rho

pytestmark = pytest.mark.gpu


def hist(rows):
    out = {}
    for r in rows:
        k = tuple(int(x) for x in r)
        out[k] = out.get(k, 0) + 1
    return out


@pytest.mark.parametrize("case", ["ket12", "rho5", "qudits"])
def test_sample_draws_match_oracle(ctx, case):
    import qpp_b200 as qb
    rng = np.random.default_rng(5)
    if case == "ket12":
        dims, x, tgt = [2] * 12, gaussian_ket(rng, 2 ** 12), [3, 0, 7]
    elif case == "rho5":
        dims, x, tgt = [2] * 5, random_rho(rng, 32, 4), [4, 1]
    else:
        dims, x, tgt = [3, 2, 3], gaussian_ket(rng, 18), [2, 0]
    s = qb.State.from_numpy(ctx, x, dims)
    got = s.sample_draws(tgt, 3000, seed=11)
    want = orc.sample(x, tgt, dims, 3000, seed=11)
    assert np.array_equal(got, want)
    counts = s.sample(tgt, 3000, seed=11)
    assert counts == hist(want)
    s.free()


def test_sample_with_given_uniforms_and_errors(ctx):
    import qpp_b200 as qb
    x = np.array([0.6, 0, 0, 0.8j])
    s = qb.State.from_numpy(ctx, x, [2, 2])
    got = s.sample_draws([0, 1], 4, u=[0.0, 0.35, 0.37, 0.99])
    assert got.tolist() == [[0, 0], [0, 0], [1, 1], [1, 1]]
    with pytest.raises(qb.OutOfRange):
        s.sample_draws([0], 0)
    with pytest.raises(qb.SubsysMismatchDims):
        s.sample_draws([2], 5)
    with pytest.raises(qb.SubsysMismatchDims):
        s.sample_draws([1, 1], 5)
    s.free()


@pytest.mark.parametrize("case,destructive,forced", [
    ("ket", True, None), ("ket", False, None), ("ket", True, [1, 0, 1]),
    ("rho_small", True, None), ("rho_small", False, None),
    ("rho_large", True, None), ("rho_large", False, [0, 1, 1])])
def test_measure_seq_matches_oracle(ctx, case, destructive, forced):
    import qpp_b200 as qb
    rng = np.random.default_rng(7)
    if case == "ket":
        n, x = 9, gaussian_ket(rng, 2 ** 9)
    elif case == "rho_small":
        n, x = 6, random_rho(rng, 64, 8)
    else:
        n, x = 11, random_rho(rng, 2 ** 11, 4)
    dims, tgt = [2] * n, [5, 1, 3]
    s = qb.State.from_numpy(ctx, x, dims)
    res, ps, out = s.measure_seq(tgt, destructive=destructive, seed=23, forced=forced)
    ores, ops_, ostate, odims = orc.measure_seq(x, tgt, dims, destructive=destructive,
                                                forced=forced, seed=23)
    assert res == ores
    assert np.allclose(ps, ops_, rtol=1e-12, atol=0)
    assert out.dims == (odims if odims else [1])
    got = out.numpy()
    assert np.max(np.abs(got - ostate)) <= 1e-12 * max(1.0, np.max(np.abs(ostate)))
    assert np.array_equal(s.numpy(), np.asarray(x).reshape(s.numpy().shape))  # unchanged
    out.free()
    s.free()


# ------------------------------------------------------------ engines
def _gates(qb, rng, c, n, layers):
    steps = []
    for _ in range(layers):
        for q in range(n):
            U = haar_unitary(rng, 2)
            c.gate(U, [q])
            steps.append((U, [q]))
        for q in range(0, n - 1, 2):
            U = haar_unitary(rng, 4)
            c.gate(U, [q, q + 1])
            steps.append((U, [q, q + 1]))
    return steps


def _evolve(steps, n):
    x = np.zeros(2 ** n, dtype=np.complex128)
    x[0] = 1
    for U, t in steps:
        x = orc.apply(x, U, t, [2] * n)
    return x


def test_execute_reps_samples_in_qpp_rng_order(ctx):
    import qpp_b200 as qb
    rng = np.random.default_rng(3)
    n, reps, seed = 6, 400, 5
    c = qb.Circuit(n, 2, n)
    steps = _gates(qb, rng, c, n, 2)
    c.measure(list(range(n)), 0, destructive=False)
    e = qb.Engine(ctx, c).set_seed(seed).execute(reps)
    psi = _evolve(steps, n)
    # draw 0: rep 0's sample (unused); draw 1: rep 0's measurement step;
    # draws 2..reps: the sampled repetitions
    draws = orc.sample(psi, list(range(n)), [2] * n, reps + 1, seed=seed)
    assert e.get_stats() == hist(draws[1:])
    assert tuple(e.get_dits()[0]) == tuple(int(v) for v in draws[1])


def test_execute_reps_canonical_reordering(ctx):
    import qpp_b200 as qb
    rng = np.random.default_rng(4)
    U, V = haar_unitary(rng, 2), haar_unitary(rng, 2)
    c = qb.Circuit(2, 2, 2)
    c.gate(U, [0]).measure([0], 0, destructive=False).gate(V, [1]).measure([1], 1, destructive=False)
    reps, seed = 300, 9
    e = qb.Engine(ctx, c).set_seed(seed).execute(reps)
    # canonical form [U0, V1, m0, m1]: the samples come from the state after
    # both gates; draws 1 and 2 belong to rep 0's two measurement steps
    psi = _evolve([(U, [0]), (V, [1])], 2)
    draws = orc.sample(psi, [0, 1], [2, 2], reps + 2, seed=seed)
    want = hist(draws[3:])
    d0 = tuple(e.get_dits()[0])
    want[d0] = want.get(d0, 0) + 1
    assert e.get_stats() == want


def test_execute_reps_keeps_the_first_repetition(ctx):
    import qpp_b200 as qb
    rng = np.random.default_rng(6)
    U, V = haar_unitary(rng, 4), haar_unitary(rng, 2)
    c = qb.Circuit(2, 2, 1)
    # a gate after the measurement on the same qubit: no sampling form
    c.gate(U, [0, 1]).measure([0], 0, destructive=False).gate(V, [0])
    for seed in (1, 2, 3):
        a = qb.Engine(ctx, c).set_seed(seed).execute(7)
        b = qb.Engine(ctx, c).set_seed(seed).execute(1)
        assert a.get_dits() == b.get_dits()
        assert np.array_equal(a.get_state().numpy(), b.get_state().numpy())
        assert sum(a.get_stats().values()) == 7
        assert len(a.get_record()[0]) == 7


def test_execute_continues_from_the_current_state(ctx):
    import qpp_b200 as qb
    rng = np.random.default_rng(8)
    U = haar_unitary(rng, 4)
    c = qb.Circuit(2)
    c.gate(U, [0, 1])
    e = qb.Engine(ctx, c).execute().execute()
    psi = _evolve([(U, [0, 1]), (U, [0, 1])], 2)
    assert np.max(np.abs(e.get_state().numpy() - psi)) < 1e-13
    assert e.get_stats() == {}  # nothing measured
    e.reset().execute()
    assert np.max(np.abs(e.get_state().numpy() - _evolve([(U, [0, 1])], 2))) < 1e-13


def test_statistics_accumulate_until_reset(ctx):
    import qpp_b200 as qb
    c = qb.Circuit(1, 2, 1)
    c.gate(np.array([[1, 1], [1, -1]]) / np.sqrt(2), [0]).measure([0], 0)
    e = qb.Engine(ctx, c).set_seed(1)
    e.execute(10)
    e.reset(reset_stats=False).execute(5)
    assert sum(e.get_stats().values()) == 15
    e.reset().execute(3)
    assert sum(e.get_stats().values()) == 3


def test_set_state_checks_size_and_kind(ctx):
    import qpp_b200 as qb
    c = qb.Circuit(3)
    e = qb.Engine(ctx, c)
    with pytest.raises(qb.DimsNotEqual):
        e.set_state(qb.State(ctx, qb.KET, [2, 2]))
    with pytest.raises(qb.TypeMismatch):
        e.set_state(qb.State(ctx, qb.RHO, [2, 2, 2]))


# ------------------------------------------- general measurements
def _close(got, want, tol=1e-12):
    got, want = np.asarray(got), np.asarray(want)
    assert got.shape == want.shape
    assert np.max(np.abs(got - want)) <= tol * max(1.0, np.max(np.abs(want)))


@pytest.mark.parametrize("kind,destructive", [("ket", True), ("ket", False), ("rho", True),
                                              ("rho", False)])
def test_measure_kraus_matches_oracle(ctx, kind, destructive):
    import qpp_b200 as qb
    from tests.qpp_helpers import depolarizing_kraus
    rng = np.random.default_rng(11)
    dims = [2] * 7
    x = gaussian_ket(rng, 128) if kind == "ket" else random_rho(rng, 128, 4)
    Ks = [np.kron(a, b) for a in depolarizing_kraus(0.3) for b in depolarizing_kraus(0.2)]
    Ks = Ks[:5] + [np.zeros((4, 4))]  # a zero-probability outcome too
    s = qb.State.from_numpy(ctx, x, dims)
    r, p, outs = s.measure_kraus(Ks, [5, 2], destructive=destructive, seed=4)
    orr, op_, oouts = orc.measure_kraus(x, Ks, [5, 2], dims, destructive=destructive, seed=4)
    assert r == orr
    assert np.allclose(p, op_, rtol=1e-12, atol=1e-15)
    for g, w in zip(outs, oouts):
        assert (g is None) == (w is None)
        if g is not None:
            _close(g.numpy(), w)
            g.free()
    s.free()


@pytest.mark.parametrize("kind,destructive", [("ket", True), ("ket", False), ("rho", True)])
def test_measure_basis_matches_oracle(ctx, kind, destructive):
    import qpp_b200 as qb
    rng = np.random.default_rng(12)
    dims = [2, 3, 2, 2]
    D = 24
    x = gaussian_ket(rng, D) if kind == "ket" else random_rho(rng, D, 3)
    V = haar_unitary(rng, 6)[:, :4]  # 4 of 6 basis vectors of the (1, 2) targets
    s = qb.State.from_numpy(ctx, x, dims)
    r, p, outs = s.measure_basis(V, [1, 2], destructive=destructive, seed=9)
    orr, op_, oouts = orc.measure_basis(x, V, [1, 2], dims, destructive=destructive, seed=9)
    assert r == orr
    assert np.allclose(p, op_, rtol=1e-12, atol=1e-15)
    for g, w in zip(outs, oouts):
        if g is not None:
            _close(g.numpy().reshape(np.asarray(w).shape), w)
            g.free()
    s.free()


@pytest.mark.parametrize("kind", ["ket", "rho"])
def test_reset_and_discard_match_oracle(ctx, kind):
    import qpp_b200 as qb
    rng = np.random.default_rng(13)
    dims = [2] * 6
    x = gaussian_ket(rng, 64) if kind == "ket" else random_rho(rng, 64, 4)
    s = qb.State.from_numpy(ctx, x, dims)
    for seed in (1, 2, 3):
        g = s.reset([4, 1], seed=seed)
        _close(g.numpy(), orc.reset(x, [4, 1], dims, seed=seed))
        g.free()
        g = s.discard([4, 1], seed=seed)
        _close(g.numpy(), orc.discard(x, [4, 1], dims, seed=seed))
        assert g.dims == [2] * 4
        g.free()
    s.free()


def test_general_measurement_errors(ctx):
    import qpp_b200 as qb
    s = qb.State(ctx, qb.KET, [2, 2], qb.C128)
    with pytest.raises(qb.MatrixMismatchSubsys):
        s.measure_kraus([np.eye(2)], [0, 1])
    with pytest.raises(qb.SubsysMismatchDims):
        s.measure_basis(np.eye(2), [2])
    with pytest.raises(qb.SubsysMismatchDims):
        s.reset([0, 0])
    s.free()
