"""Density-matrix subsystem ops at the full 12-qubit size (4096 x 4096).

rho = W W^+ / tr(W W^+) from a 4096 x 64 complex Gaussian W (rank 64). Each
step applies the 2-qubit channel (depolarising p=0.01 composed with
amplitude damping gamma=0.02 on each qubit, 16 Kraus operators) on a random
pair, then ptrace over a random 6-subset, ptranspose over a random 6-subset
and syspermute by a random permutation. Checked through properties that do
not need the oracle at this size:
  * the channel preserves the trace (1e-12) and Hermiticity (1e-12);
  * ptranspose twice over the same subset and syspermute followed by the
    inverse permutation return the input bit for bit;
  * ptrace over A then B equals ptrace over A u B (1e-12), and the reduced
    state has unit trace;
and, at 8 qubits, against the oracle step by step (1e-12). The mixed
dimension variant (dims [3,3,2,2,3,2,2,3], Haar 3x3 and 6x6 gates) runs
against the oracle at full size.
"""
import numpy as np
import pytest

from oracle import oracle as orc
from tests.qpp_helpers import haar_unitary, random_rho

pytestmark = pytest.mark.gpu


def _inv(perm):
    inv = [0] * len(perm)
    for i, p in enumerate(perm):
        inv[p] = i
    return inv


def test_rho_12q_steps_properties(ctx):
    import qpp_b200 as qb
    from qpp_b200.serving import pair_channel
    rng = np.random.default_rng(12)
    n, D = 12, 4096
    W = rng.standard_normal((D, 64)) + 1j * rng.standard_normal((D, 64))
    rho = W @ W.conj().T
    rho /= np.trace(rho).real
    s = qb.State.from_numpy(ctx, rho, [2] * n)
    Ks = pair_channel()
    for step in range(20):
        pair = [int(x) for x in rng.choice(n, size=2, replace=False)]
        s.apply_kraus(Ks, pair)
        tr = s.trace()
        assert abs(tr - 1) < 1e-12
        A = [int(x) for x in rng.choice(n, size=6, replace=False)]
        red = s.ptrace(A)
        assert abs(red.trace() - 1) < 1e-12
        T = [int(x) for x in rng.choice(n, size=6, replace=False)]
        pt = s.ptranspose(T)
        back = pt.ptranspose(T).numpy()
        perm = [int(x) for x in rng.permutation(n)]
        sp = s.syspermute(perm)
        s2 = sp.syspermute(_inv(perm))
        cur = s.numpy()
        assert np.array_equal(back, cur)
        assert np.array_equal(s2.numpy(), cur)
        s = sp  # rho <- syspermute(rho, perm), as in the workload
    cur = s.numpy()
    assert np.max(np.abs(cur - cur.conj().T)) < 1e-12
    A, B = [0, 3, 5], [7, 10]
    two = s.ptrace(A)
    rest = [q for q in range(n) if q not in A]
    via = two.ptrace([rest.index(b) for b in B]).numpy()
    assert np.max(np.abs(via - s.ptrace(A + B).numpy())) < 1e-12


def test_rho_8q_steps_match_oracle(ctx):
    import qpp_b200 as qb
    from qpp_b200.serving import pair_channel
    rng = np.random.default_rng(8)
    n = 8
    rho = random_rho(rng, 2 ** n, 16)
    ref = rho.copy()
    s = qb.State.from_numpy(ctx, rho, [2] * n)
    Ks = pair_channel()
    for step in range(6):
        pair = [int(x) for x in rng.choice(n, size=2, replace=False)]
        s.apply_kraus(Ks, pair)
        ref = orc.apply_kraus(ref, Ks, pair, [2] * n)
        A = [int(x) for x in rng.choice(n, size=4, replace=False)]
        assert np.max(np.abs(s.ptrace(A).numpy() - orc.ptrace(ref, A, [2] * n))) < 1e-12
        perm = [int(x) for x in rng.permutation(n)]
        s = s.syspermute(perm)
        ref = orc.syspermute(ref, perm, [2] * n)
        assert np.max(np.abs(s.numpy() - ref)) / np.max(np.abs(ref)) < 1e-12


def test_mixed_dims_full_size(ctx):
    import qpp_b200 as qb
    rng = np.random.default_rng(1296)
    dims = [3, 3, 2, 2, 3, 2, 2, 3]
    D = int(np.prod(dims))
    rho = random_rho(rng, D, 64)
    ref = rho.copy()
    s = qb.State.from_numpy(ctx, rho, dims)
    for step in range(3):
        t3 = int(rng.choice([0, 1, 4, 7]))
        U = haar_unitary(rng, 3)
        s.apply(U, [t3])
        ref = orc.apply(ref, U, [t3], dims)
        pair = [int(rng.choice([0, 1, 4, 7])), int(rng.choice([2, 3, 5, 6]))]
        U6 = haar_unitary(rng, 6)
        s.apply(U6, pair)
        ref = orc.apply(ref, U6, pair, dims)
        half = [int(x) for x in rng.choice(8, size=4, replace=False)]
        assert np.max(np.abs(s.ptrace(half).numpy() - orc.ptrace(ref, half, dims))) < 1e-12
        assert np.array_equal(s.ptranspose(half).numpy(), orc.ptranspose(s.numpy(), half, dims))
        perm = [int(x) for x in rng.permutation(8)]
        sp = s.syspermute(perm)
        assert np.array_equal(sp.numpy(), orc.syspermute(s.numpy(), perm, dims))
    assert np.max(np.abs(s.numpy() - ref)) / np.max(np.abs(ref)) < 1e-12


def _random_channel(rng, d, nk):
    """nk Kraus operators of a random d-dimensional channel (sum K^+ K = I)."""
    G = rng.standard_normal((nk * d, d)) + 1j * rng.standard_normal((nk * d, d))
    Q, _ = np.linalg.qr(G)
    return [Q[i * d:(i + 1) * d, :] for i in range(nk)]


@pytest.mark.parametrize("prec", ["c128", "c64"])
def test_two_qubit_channel_product_and_general(ctx, prec):
    """A product of two one-qubit channels on a qubit pair has a superoperator
    that factors as A (x) B; the library then applies the two 4 x 4 factors in
    one pass. Both that path (product channel, 3 x 2 Kraus operators) and the
    16 x 16 path (a random two-qubit channel, 5 operators) match the oracle
    within 1e-12 in complex128 (2e-5 in complex64), on pairs in both orders
    and with the pair straddling the matrix's row and column digits."""
    import qpp_b200 as qb
    tol = 1e-12 if prec == "c128" else 2e-5
    P = qb.C128 if prec == "c128" else qb.C64
    rng = np.random.default_rng(5 if prec == "c128" else 6)
    n = 6
    dims = [2] * n
    for pair in ([1, 4], [5, 0], [2, 3]):
        KA, KB = _random_channel(rng, 2, 3), _random_channel(rng, 2, 2)
        prod = [np.kron(a, b) for a in KA for b in KB]
        gen = _random_channel(rng, 4, 5)
        for Ks in (prod, gen):
            x = random_rho(rng, 2 ** n, 5)
            s = qb.State.from_numpy(ctx, x, dims, P)
            s.apply_kraus(Ks, pair)
            ref = orc.apply_kraus(x, Ks, pair, dims)
            got = s.numpy()
            assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) < tol, (pair, len(Ks))
