"""Known-answer tests of Quantum++'s own suite, restated.

Every case cites the reference test it restates. Each runs on two backends
with qpp's value-semantics signatures: the CPU oracle (pins the restatement
against the reference's KATs) and the GPU C-ABI (qgpu_host_* entry points,
marked gpu). Tolerances are the reference's (1e-5, 1e-10, 1e-12, or exact
where the reference uses EXPECT_EQ).
"""
import numpy as np
import pytest

from tests.qpp_helpers import (CNOT, TOF, H, X, Xd, Y, Z, dense_gate, gaussian_ket,
                               haar_unitary, ket_from_bits, mket, mprj, prj, random_rho)

BACKENDS = ["oracle", pytest.param("gpu", marks=pytest.mark.gpu)]


class _OracleBackend:
    def __init__(self):
        from oracle import oracle
        self.m = oracle

    def apply(self, s, A, t, dims):
        return self.m.apply(s, A, t, dims)

    def applyCTRL(self, s, A, c, t, dims, shift=None):
        return self.m.applyCTRL(s, A, c, t, dims, shift)

    def applyCTRL_fan(self, s, A, c, t, dims, shift=None):
        return self.m.applyCTRL_fan(s, A, c, t, dims, shift)

    def apply_kraus(self, s, Ks, t, dims):
        return self.m.apply_kraus(s, Ks, t, dims)

    def ptrace(self, s, t, dims):
        return self.m.ptrace(s, t, dims)

    def ptranspose(self, s, t, dims):
        return self.m.ptranspose(s, t, dims)

    def syspermute(self, s, p, dims):
        return self.m.syspermute(s, p, dims)

    def measure_seq(self, s, t, dims, destructive):
        res, probs, out, _ = self.m.measure_seq(s, t, dims, destructive=destructive)
        return res, probs, out


class _GpuBackend:
    def __init__(self, ctx):
        import qpp_b200 as qb
        self.qb, self.ctx = qb, ctx

    def apply(self, s, A, t, dims):
        return self.qb.apply(s, A, t, dims, ctx=self.ctx)

    def applyCTRL(self, s, A, c, t, dims, shift=None):
        return self.qb.applyCTRL(s, A, c, t, dims, shift, ctx=self.ctx)

    def applyCTRL_fan(self, s, A, c, t, dims, shift=None):
        return self.qb.applyCTRL_fan(s, A, c, t, dims, shift, ctx=self.ctx)

    def apply_kraus(self, s, Ks, t, dims):
        return self.qb.apply_kraus(s, Ks, t, dims, ctx=self.ctx)

    def ptrace(self, s, t, dims):
        return self.qb.ptrace(s, t, dims, ctx=self.ctx)

    def ptranspose(self, s, t, dims):
        return self.qb.ptranspose(s, t, dims, ctx=self.ctx)

    def syspermute(self, s, p, dims):
        return self.qb.syspermute(s, p, dims, ctx=self.ctx)

    def measure_seq(self, s, t, dims, destructive):
        st = self.qb.State.from_numpy(self.ctx, s, dims)
        res, probs, out = st.measure_seq(t, destructive=destructive)
        x = out.numpy()
        out.free()
        st.free()
        return res, probs, x


@pytest.fixture(params=BACKENDS)
def be(request):
    if request.param == "oracle":
        return _OracleBackend()
    return _GpuBackend(request.getfixturevalue("ctx"))


def _norm(a):
    return float(np.linalg.norm(np.asarray(a).reshape(-1)))


# ----------------------------------------------- operations.cpp:16-74
def test_apply_qudits_1qubit(be):
    psi = mket([1])
    assert np.array_equal(be.apply(psi, X, [0], [2]), mket([0]))
    assert np.array_equal(be.apply(psi, Y, [0], [2]), -1j * mket([0]))
    assert np.array_equal(be.apply(psi, Z, [0], [2]), -mket([1]))
    r = be.apply(psi, H, [0], [2])
    assert _norm(r - (mket([0]) - mket([1])) / np.sqrt(2)) < 1e-5


def test_apply_qudits_2qubits(be):
    psi = 0.8 * ket_from_bits("00") + 0.6 * ket_from_bits("11")
    b = ket_from_bits
    assert np.array_equal(be.apply(psi, X, [1], [2, 2]), 0.8 * b("01") + 0.6 * b("10"))
    assert np.array_equal(be.apply(psi, Y, [1], [2, 2]), 0.8j * b("01") - 0.6j * b("10"))
    assert np.array_equal(be.apply(psi, Z, [1], [2, 2]), 0.8 * b("00") - 0.6 * b("11"))
    assert np.array_equal(be.apply(psi, CNOT, [0, 1], [2, 2]), 0.8 * b("00") + 0.6 * b("10"))
    assert np.array_equal(be.apply(psi, CNOT, [1, 0], [2, 2]), 0.8 * b("00") + 0.6 * b("01"))
    assert np.array_equal(be.apply(psi, np.kron(Z, Z), [0, 1], [2, 2]), psi)


def test_apply_qudits_4qubits(be):
    b = ket_from_bits
    psi = 0.8 * b("0000") + 0.6 * b("1111")
    XZ = np.kron(X, Z)
    assert np.array_equal(be.apply(psi, XZ, [1, 2], [2] * 4), 0.8 * b("0100") - 0.6 * b("1011"))
    assert np.array_equal(be.apply(psi, XZ, [2, 1], [2] * 4), 0.8 * b("0010") - 0.6 * b("1101"))
    assert np.array_equal(be.apply(psi, TOF, [1, 2, 0], [2] * 4), 0.8 * b("0000") + 0.6 * b("0111"))


def test_apply_qudits_qutrits(be):
    d = 3
    psi = mket([0, 0], d) + mket([1, 0], d) / np.sqrt(2)
    r = be.apply(psi, Xd(d), [0], [d, d])
    exp = mket([1, 0], d) + mket([2, 0], d) / np.sqrt(2)
    assert _norm(r - exp) < 1e-5
    rho = 0.6 * prj(mket([0, 0], d) + mket([1, 0], d) / np.sqrt(2)) + \
        0.4 * prj(mket([0, 1], d) + mket([1, 1], d) / np.sqrt(2))
    r = be.apply(rho, Xd(d), [0], [d, d])
    exp = 0.6 * prj(mket([1, 0], d) + mket([2, 0], d) / np.sqrt(2)) + \
        0.4 * prj(mket([1, 1], d) + mket([2, 1], d) / np.sqrt(2))
    assert _norm(r - exp) < 1e-5


# ---------------------------------------------- operations.cpp:101-162
def test_applyCTRL_qudits(be):
    d, n = 3, 4
    dims = [d] * n
    ctrl, target = [0, 2], [1, 3]
    XX = np.kron(Xd(3), Xd(3))
    r = be.applyCTRL(mket([2, 1, 2, 1], d), XX, ctrl, target, dims)
    assert _norm(r - mket([2, 0, 2, 0], d)) < 1e-5
    r = be.applyCTRL(mket([2, 1, 1, 1], d), XX, ctrl, target, dims, [1, 2])
    assert _norm(r - mket([2, 1, 1, 1], d)) < 1e-5
    r = be.applyCTRL(prj(mket([2, 0, 2, 0], d)), XX, ctrl, target, dims)
    assert _norm(r - mprj([2, 2, 2, 2], d)) < 1e-5
    r = be.applyCTRL(prj(mket([1, 0, 0, 0], d)), XX, ctrl, target, dims, [1, 2])
    assert _norm(r - mprj([1, 2, 0, 2], d)) < 1e-5
    rng = np.random.default_rng(101)
    psi = gaussian_ket(rng, d ** n)
    U = haar_unitary(rng, 9)
    A = be.applyCTRL(psi, U, ctrl, target, dims)
    B = be.applyCTRL(prj(psi), U, ctrl, target, dims)
    assert _norm(prj(A) - B) < 1e-5


# ---------------------------------------------- operations.cpp:176-230
def test_applyCTRL_fan_qudits(be):
    d, n = 3, 4
    dims = [d] * n
    ctrl, target = [0, 2], [1, 3]
    r = be.applyCTRL_fan(mket([2, 1, 2, 1], d), Xd(3), ctrl, target, dims)
    assert _norm(r - mket([2, 0, 2, 0], d)) < 1e-5
    r = be.applyCTRL_fan(mket([2, 1, 1, 1], d), Xd(3), ctrl, target, dims, [1, 2])
    assert _norm(r - mket([2, 1, 1, 1], d)) < 1e-5
    r = be.applyCTRL_fan(prj(mket([2, 0, 2, 0], d)), Xd(3), ctrl, target, dims)
    assert _norm(r - mprj([2, 2, 2, 2], d)) < 1e-5
    r = be.applyCTRL_fan(prj(mket([1, 0, 0, 0], d)), Xd(3), ctrl, target, dims, [1, 2])
    assert _norm(r - mprj([1, 2, 0, 2], d)) < 1e-5
    rng = np.random.default_rng(176)
    psi = gaussian_ket(rng, d ** n)
    U = haar_unitary(rng, d)
    A = be.applyCTRL_fan(psi, U, ctrl, target, dims)
    B = be.applyCTRL_fan(prj(psi), U, ctrl, target, dims)
    assert _norm(prj(A) - B) < 1e-5


# ---------------------------------------------- operations.cpp:237-397
def test_applyCTRL_fan_qubits(be):
    n, m = 6, 3
    ctrl, target = list(range(m)), list(range(m, 2 * m))
    dims = [2] * n
    # A) controls |1>, targets |0> -> all targets flip
    midx = [1] * m + [0] * m
    out = be.applyCTRL_fan(mket(midx), X, ctrl, target, dims)
    assert _norm(out - mket([1] * n)) < 1e-12
    # B) first and last control negated: pattern (0, 1, 0) matches
    shift = [1, 0, 1]
    midx = [0, 1, 0, 0, 0, 0]
    out = be.applyCTRL_fan(mket(midx), X, ctrl, target, dims, shift)
    assert _norm(out - mket([0, 1, 0, 1, 1, 1])) < 1e-12
    # C) broken control -> unchanged
    midx = [0, 0, 0, 0, 0, 0]
    out = be.applyCTRL_fan(mket(midx), X, ctrl, target, dims, shift)
    assert _norm(out - mket(midx)) < 1e-12
    # D) density matrix, no shift
    rho = be.applyCTRL_fan(prj(mket([1] * m + [0] * m)), X, ctrl, target, dims)
    assert _norm(rho - mprj([1] * n)) < 1e-12
    # E) density matrix, with shift
    rho = be.applyCTRL_fan(prj(mket([0, 1, 0, 0, 0, 0])), X, ctrl, target, dims, shift)
    assert _norm(rho - mprj([0, 1, 0, 1, 1, 1])) < 1e-12
    # F) random ket vs density consistency
    rng = np.random.default_rng(237)
    psi = gaussian_ket(rng, 2 ** n)
    U = haar_unitary(rng, 2)
    A = be.applyCTRL_fan(psi, U, ctrl, target, dims)
    B = be.applyCTRL_fan(prj(psi), U, ctrl, target, dims)
    assert _norm(prj(A) - prj(A).conj().T) < 1e-10
    assert _norm(B - B.conj().T) < 1e-10
    assert _norm(prj(A) - B) < 1e-10


# --------------------------------------------- classes/gates.cpp:170-207
def test_gate_vs_apply_qudits(be):
    d, n = 3, 4
    dims = [d] * n
    psi = mket([1, 1, 1, 1], d)
    U = np.kron(Xd(d), Xd(d) @ Xd(d))
    assert _norm(be.apply(psi, U, [1, 3], dims) - mket([1, 2, 1, 0], d)) < 1e-5
    assert _norm(be.apply(psi, U, [3, 1], dims) - mket([1, 0, 1, 2], d)) < 1e-5
    rng = np.random.default_rng(170)
    U = haar_unitary(rng, d * d)
    assert _norm(dense_gate(U, [1, 3], dims) @ psi - be.apply(psi, U, [1, 3], dims)) < 1e-5
    assert _norm(dense_gate(U, [3, 1], dims) @ psi - be.apply(psi, U, [1, 3], dims)) > 1e-5


def test_gate_vs_apply_qubits(be):
    psi = mket([1, 1, 1, 1])
    dims = [2] * 4
    assert _norm(be.apply(psi, CNOT, [1, 3], dims) - mket([1, 1, 1, 0])) < 1e-5
    assert _norm(be.apply(psi, CNOT, [3, 1], dims) - mket([1, 0, 1, 1])) < 1e-5
    rng = np.random.default_rng(171)
    U = haar_unitary(rng, 4)
    assert _norm(dense_gate(U, [1, 3], dims) @ psi - be.apply(psi, U, [1, 3], dims)) < 1e-5
    assert _norm(dense_gate(U, [3, 1], dims) @ psi - be.apply(psi, U, [1, 3], dims)) > 1e-5


# ------------------------------------------------ entropies.cpp:103-108
def _entropy(rho):
    ev = np.linalg.eigvalsh((rho + rho.conj().T) / 2)
    ev = ev[ev > 1e-14]
    return float(-(ev * np.log2(ev)).sum())


def test_syspermute_mutual_information(be):
    # MES(3) (x) rho_2 (x) rho_2, subsystems permuted {0, 2, 1, 3}: the
    # MES halves end up at positions 0 and 2, I(0:2) = 2 log2 3.
    rng = np.random.default_rng(103)
    mes = np.zeros(9, dtype=np.complex128)
    for i in range(3):
        mes[i * 3 + i] = 1 / np.sqrt(3)
    rho = np.kron(prj(mes), np.kron(random_rho(rng, 2, 2), random_rho(rng, 2, 2)))
    rho = be.syspermute(rho, [0, 2, 1, 3], [3, 3, 2, 2])
    dims = [3, 2, 3, 2]
    rA = be.ptrace(rho, [1, 2, 3], dims)
    rB = be.ptrace(rho, [0, 1, 3], dims)
    rAB = be.ptrace(rho, [1, 3], dims)
    mi = _entropy(rA) + _entropy(rB) - _entropy(rAB)
    assert abs(mi - 2 * np.log2(3)) < 1e-5


# --------------------------------------------- entanglement.cpp:108-111
def _lognegativity(be, rho, dims):
    pt = be.ptranspose(rho, [0], dims)
    return float(np.log2(np.abs(np.linalg.eigvalsh((pt + pt.conj().T) / 2)).sum()))


def test_lognegativity_additivity(be):
    rng = np.random.default_rng(108)
    rho, sigma = random_rho(rng, 4, 4), random_rho(rng, 4, 4)
    lhs = _lognegativity(be, be.syspermute(np.kron(rho, sigma), [0, 2, 1, 3], [2, 2, 2, 2]), [4, 4])
    rhs = _lognegativity(be, rho, [2, 2]) + _lognegativity(be, sigma, [2, 2])
    assert abs(lhs - rhs) < 1e-5


# ------------------------------------ Kraus channel: trace preservation
def test_kraus_channel_trace_and_dense(be):
    from tests.qpp_helpers import amplitude_damping_kraus, depolarizing_kraus
    rng = np.random.default_rng(476)
    dims = [2, 3, 2]
    rho = random_rho(rng, 12, 3)
    Ks = [np.kron(a, b) for a in depolarizing_kraus(0.01) for b in amplitude_damping_kraus(0.02)]
    out = be.apply_kraus(rho, Ks, [2, 0], dims)
    assert abs(np.trace(out) - 1) < 1e-12
    ref = sum(dense_gate(K, [2, 0], dims) @ rho @ dense_gate(K, [2, 0], dims).conj().T for K in Ks)
    assert np.max(np.abs(out - ref)) < 1e-12


# unit_tests/tests/instruments.cpp:102-160 (qpp_measure_seq, Qudits)
def test_measure_seq_qudits(be):
    dims = [2, 2, 3, 2, 3, 2]
    mask = [0, 1, 2, 1, 2, 0]
    psi, rho = mket(mask, dims), mprj(mask, dims)
    ms, ps, out = be.measure_seq(psi, [4, 2, 3, 0], dims, True)
    assert ms == [2, 2, 1, 0] and ps == [1, 1, 1, 1]
    assert _norm(np.asarray(out).reshape(-1) - mket([1, 0], [2, 2])) < 1e-5
    ms, ps, out = be.measure_seq(rho, [4, 2, 3, 0], dims, True)
    assert ms == [2, 2, 1, 0] and ps == [1, 1, 1, 1]
    assert _norm(out - mprj([1, 0], [2, 2])) < 1e-5
    ms, ps, out = be.measure_seq(psi, [4, 2, 3, 0], dims, False)
    assert ms == [2, 2, 1, 0] and ps == [1, 1, 1, 1]
    assert _norm(np.asarray(out).reshape(-1) - psi) < 1e-5
    ms, ps, out = be.measure_seq(psi, [3, 0, 4, 2], dims, False)
    assert ms == [1, 0, 2, 2] and ps == [1, 1, 1, 1]
    assert _norm(np.asarray(out).reshape(-1) - psi) < 1e-5
    ms, ps, out = be.measure_seq(rho, [3, 0, 4, 2], dims, False)
    assert ms == [1, 0, 2, 2] and ps == [1, 1, 1, 1]
    assert _norm(out - rho) < 1e-5
