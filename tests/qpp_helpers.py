"""Gate and state constructors of Quantum++ restated in numpy for the tests.

Gates follow include/qpp/classes/gates.hpp (X, Y, Z, H, CNOT, TOF, Xd, Zd, Fd);
mket/mprj/prj follow include/qpp/functions.hpp:1576-1700. The random inputs
(Haar unitaries, Gaussian kets, rank-r density matrices) come from this
project's own seeded generator (numpy PCG64), since qpp's randU/randket draw
from an unseeded mt19937 (random.hpp:257-412).
"""
import numpy as np

X = np.array([[0, 1], [1, 0]], dtype=np.complex128)
Y = np.array([[0, -1j], [1j, 0]], dtype=np.complex128)
Z = np.array([[1, 0], [0, -1]], dtype=np.complex128)
H = np.array([[1, 1], [1, -1]], dtype=np.complex128) / np.sqrt(2)
Id2 = np.eye(2, dtype=np.complex128)
CNOT = np.eye(4, dtype=np.complex128)[[0, 1, 3, 2]]
TOF = np.eye(8, dtype=np.complex128)[[0, 1, 2, 3, 4, 5, 7, 6]]


def Zd(D):
    if D == 2:
        return Z.copy()
    w = np.exp(2j * np.pi / D)
    return np.diag([w ** i for i in range(D)]).astype(np.complex128)


def Fd(D):
    w = np.exp(2j * np.pi / D)
    return np.array([[w ** (j * k) for k in range(D)] for j in range(D)]) / np.sqrt(D)


def Xd(D):
    if D == 2:
        return X.copy()
    F = Fd(D)
    return np.linalg.inv(F) @ Zd(D) @ F


def mket(mask, d=2):
    dims = list(d) if isinstance(d, (list, tuple)) else [d] * len(mask)
    D = int(np.prod(dims))
    i = 0
    for m, dd in zip(mask, dims):
        i = i * dd + m
    v = np.zeros(D, dtype=np.complex128)
    v[i] = 1
    return v


def prj(psi):
    psi = np.asarray(psi).reshape(-1)
    return np.outer(psi, psi.conj())


def mprj(mask, d=2):
    return prj(mket(mask, d))


def ket_from_bits(s):
    """'0110' -> |0110> (qubits, big-endian)."""
    return mket([int(c) for c in s], 2)


def haar_unitary(rng, D):
    """Haar-distributed unitary: QR of a complex Ginibre matrix with the
    phases of R's diagonal moved into Q (Mezzadri 2007)."""
    Zm = (rng.standard_normal((D, D)) + 1j * rng.standard_normal((D, D))) / np.sqrt(2)
    Q, R = np.linalg.qr(Zm)
    ph = np.diag(R) / np.abs(np.diag(R))
    return (Q * ph).astype(np.complex128)


def gaussian_ket(rng, D):
    v = rng.standard_normal(D) + 1j * rng.standard_normal(D)
    return (v / np.linalg.norm(v)).astype(np.complex128)


def random_rho(rng, D, rank):
    W = rng.standard_normal((D, rank)) + 1j * rng.standard_normal((D, rank))
    r = W @ W.conj().T
    return (r / np.trace(r).real).astype(np.complex128)


def dense_gate(U, target, dims):
    """Gates::GATE(U, target, dims) (gates.hpp:409): the full D x D operator
    of U acting on `target`, built by explicit index expansion."""
    dims = list(dims)
    n = len(dims)
    D = int(np.prod(dims))
    dt = [dims[t] for t in target]
    DA = int(np.prod(dt))
    M = np.zeros((D, D), dtype=np.complex128)
    strides = [int(np.prod(dims[i + 1:])) for i in range(n)]
    for col in range(D):
        dig = []
        c = col
        for dd in reversed(dims):
            dig.append(c % dd)
            c //= dd
        dig = dig[::-1]
        a_in = 0
        for t in target:
            a_in = a_in * dims[t] + dig[t]
        base = col - sum(dig[t] * strides[t] for t in target)
        for a_out in range(DA):
            rem = a_out
            off = 0
            for t in reversed(target):
                off += (rem % dims[t]) * strides[t]
                rem //= dims[t]
            M[base + off, col] += U[a_out, a_in]
    return M


def depolarizing_kraus(p):
    """QubitDepolarizingNoise Kraus set (noise.hpp:388-412) as operators:
    sqrt(1-p) I, sqrt(p/3) X, sqrt(p/3) Y, sqrt(p/3) Z."""
    return [np.sqrt(1 - p) * Id2, np.sqrt(p / 3) * X, np.sqrt(p / 3) * Y, np.sqrt(p / 3) * Z]


def amplitude_damping_kraus(gamma):
    """Standard amplitude damping with decay probability gamma:
    K0 = [[1, 0], [0, sqrt(1-gamma)]], K1 = [[0, sqrt(gamma)], [0, 0]].
    (qpp's QubitAmplitudeDampingNoise(g), noise.hpp:495-496, uses the
    survival parameter: its K0 carries sqrt(g), i.e. gamma_std = 1 - g.)"""
    return [np.array([[1, 0], [0, np.sqrt(1 - gamma)]], dtype=np.complex128),
            np.array([[0, np.sqrt(gamma)], [0, 0]], dtype=np.complex128)]
