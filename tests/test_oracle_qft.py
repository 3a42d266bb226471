"""The oracle's restatement of qpp::applyQFT / applyTFQ / QFT / TFQ
(operations.hpp:2565-2899), pinned by the transform's definition: the
reference's own tests for these functions are empty bodies
(unit_tests/tests/operations.cpp:399-406, :459-461, :484-486), so the pin is
the DFT identity QFT(psi) = sqrt(N) * ifft(psi) on the register spelled by the
targets (target[0] most significant), its inverse, the digit reversal that
swap=False leaves out, and U rho U^dagger on density matrices."""
import numpy as np
import pytest

from oracle import oracle as orc


def _reg_dft(psi, dims, target, inverse):
    """DFT (or its adjoint) over the target digits, target[0] most significant."""
    n = len(dims)
    a = np.asarray(psi).reshape(dims)
    rest = [q for q in range(n) if q not in target]
    a = np.transpose(a, list(target) + rest)
    N = int(np.prod([dims[t] for t in target]))
    a = a.reshape(N, -1)
    a = (np.fft.fft(a, axis=0) / np.sqrt(N)) if inverse else (np.fft.ifft(a, axis=0) * np.sqrt(N))
    a = a.reshape([dims[t] for t in target] + [dims[q] for q in rest])
    inv = np.argsort(list(target) + rest)
    return np.transpose(a, inv).reshape(-1)


def _reverse(psi, dims, target):
    """Digit target[i] takes the value of digit target[k-1-i]."""
    n = len(dims)
    a = np.asarray(psi).reshape(dims)
    perm = list(range(n))
    k = len(target)
    for i in range(k):
        perm[target[i]] = target[k - 1 - i]
    return np.transpose(a, perm).reshape(-1)


@pytest.mark.parametrize("d,n", [(2, 1), (2, 4), (2, 6), (3, 3), (4, 2), (5, 2)])
def test_qft_equals_dft(d, n):
    rng = np.random.default_rng(d * 100 + n)
    D = d ** n
    psi = rng.normal(size=D) + 1j * rng.normal(size=D)
    psi /= np.linalg.norm(psi)
    dims = [d] * n
    for rep in range(3):
        k = n if rep == 0 else int(rng.integers(1, n + 1))
        t = [int(x) for x in rng.permutation(n)[:k]]
        if rep == 0:
            t.sort()
        ref = _reg_dft(psi, dims, t, False)
        assert np.max(np.abs(orc.applyQFT(psi, t, d) - ref)) < 1e-13
        assert np.max(np.abs(orc.applyQFT(psi, t, d, swap=False) - _reverse(ref, dims, t))) < 1e-13
        ref_i = _reg_dft(psi, dims, t, True)
        assert np.max(np.abs(orc.applyTFQ(psi, t, d) - ref_i)) < 1e-13
        # TFQ without swap is the adjoint of QFT without swap
        back = orc.applyTFQ(orc.applyQFT(psi, t, d, swap=False), t, d, swap=False)
        assert np.max(np.abs(back - psi)) < 1e-13
    assert np.max(np.abs(orc.QFT(psi, d) - _reg_dft(psi, dims, list(range(n)), False))) < 1e-13
    assert np.max(np.abs(orc.TFQ(psi, d) - _reg_dft(psi, dims, list(range(n)), True))) < 1e-13


def test_qft_on_density_matrix():
    rng = np.random.default_rng(5)
    n, d = 3, 2
    D = d ** n
    W = rng.normal(size=(D, 2)) + 1j * rng.normal(size=(D, 2))
    rho = W @ W.conj().T
    rho /= np.trace(rho)
    t = [2, 0]
    U = np.stack([orc.applyQFT(np.eye(D)[:, c], t, d) for c in range(D)], axis=1)
    got = orc.applyQFT(rho, t, d)
    assert np.max(np.abs(got - U @ rho @ U.conj().T)) < 1e-13


@pytest.mark.parametrize("call,code,where,what", [
    (lambda: orc.applyQFT(np.zeros(0), [0]), 1, "qpp::applyQFT()", "A"),
    (lambda: orc.applyQFT(np.ones(4), [0], d=1), 5, "qpp::applyQFT()", "d"),
    (lambda: orc.applyQFT(np.ones(4), [2]), 9, "qpp::applyQFT()", "dims/target"),
    (lambda: orc.applyQFT(np.ones(4), [0, 0]), 9, "qpp::applyQFT()", "dims/target"),
    (lambda: orc.applyTFQ(np.ones(6), [0]), 8, "qpp::applyTFQ()", "A/dims"),
    (lambda: orc.applyQFT(np.ones((6, 6)), [0]), 7, "qpp::applyQFT()", "A/dims"),
    (lambda: orc.applyQFT(np.ones((4, 2)), [0]), 3, "qpp::applyQFT()", "A"),
    (lambda: orc.TFQ(np.ones(6)), 8, "qpp::QFT()", "A/dims"),
    (lambda: orc.TFQ(np.ones(4), d=1), 5, "qpp::TFQ()", "d"),
])
def test_qft_errors(call, code, where, what):
    with pytest.raises(orc.OracleError) as e:
        call()
    assert (e.value.code, e.value.where, e.value.what) == (code, where, what)
