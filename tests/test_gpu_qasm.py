"""OpenQASM 2.0 programs on the device engines.

* teleportation (the circuit of the reference's
  unit_tests/tests/qasm/circuits/units/teleportation.qasm test, written out
  here as our own program): the teleported qubit ends in |0> after the
  inverse rotation for every measurement outcome, on QEngine and
  QDensityEngine;
* a random program over qelib1's gates agrees with the oracle applying the
  gates' matrices, written independently below from their definitions
  (Qiskit's U convention, Rn rotations), within 1e-12;
* reset and if: deterministic outcomes.
"""
import numpy as np
import pytest

from oracle import oracle as orc
from tests.qpp_helpers import prj

pytestmark = pytest.mark.gpu
HEAD = 'OPENQASM 2.0;\ninclude "qelib1.inc";\n'

TELEPORT = HEAD + """qreg q[3];
creg c0[1];
creg c1[1];
u3(0.3, 0.2, 0.1) q[0];
h q[1];
cx q[1], q[2];
barrier q;
cx q[0], q[1];
h q[0];
measure q[0] -> c0[0];
measure q[1] -> c1[0];
if (c0 == 1) z q[2];
if (c1 == 1) x q[2];
u3(-0.3, -0.1, -0.2) q[2];
"""


@pytest.mark.parametrize("kind", ["ket", "rho"])
def test_teleportation_program(ctx, kind):
    import qpp_b200 as qb
    c = qb.Circuit.from_qasm(TELEPORT)
    seen = set()
    for seed in range(12):
        e = qb.Engine(ctx, c, qb.KET if kind == "ket" else qb.RHO).set_seed(seed).execute()
        rho = orc.ptrace(e.get_state().numpy(), [0, 1], [2, 2, 2])
        assert np.linalg.norm(rho - prj(np.array([1, 0]))) < 1e-12
        seen.add(tuple(e.get_dits()[0]))
    assert len(seen) > 1


def U(t, p, l):
    return np.array([[np.cos(t / 2), -np.exp(1j * l) * np.sin(t / 2)],
                     [np.exp(1j * p) * np.sin(t / 2), np.exp(1j * (p + l)) * np.cos(t / 2)]])


X = np.array([[0, 1], [1, 0]], dtype=complex)
Y = np.array([[0, -1j], [1j, 0]])
Z = np.diag([1, -1]).astype(complex)
H = np.array([[1, 1], [1, -1]]) / np.sqrt(2)
S = np.diag([1, 1j])
T = np.diag([1, np.exp(1j * np.pi / 4)])


def R(t, P):
    return np.cos(t / 2) * np.eye(2) - 1j * np.sin(t / 2) * P


def ctl(M):
    out = np.eye(4, dtype=complex)
    out[2:, 2:] = M
    return out


SWAP = np.eye(4)[[0, 2, 1, 3]]
GATES = {  # name: (params, qubits, matrix)
    "u3": (3, 1, lambda a: U(*a)), "u2": (2, 1, lambda a: U(np.pi / 2, *a)),
    "u1": (1, 1, lambda a: U(0, 0, a[0])), "rx": (1, 1, lambda a: R(a[0], X)),
    "ry": (1, 1, lambda a: R(a[0], Y)), "rz": (1, 1, lambda a: R(a[0], Z)),
    "h": (0, 1, lambda a: H), "s": (0, 1, lambda a: S), "sdg": (0, 1, lambda a: S.conj().T),
    "t": (0, 1, lambda a: T), "tdg": (0, 1, lambda a: T.conj().T), "x": (0, 1, lambda a: X),
    "y": (0, 1, lambda a: Y), "z": (0, 1, lambda a: Z),
    "sx": (0, 1, lambda a: np.array([[1 + 1j, 1 - 1j], [1 - 1j, 1 + 1j]]) / 2),
    "cx": (0, 2, lambda a: ctl(X)), "cz": (0, 2, lambda a: ctl(Z)), "cy": (0, 2, lambda a: ctl(Y)),
    "ch": (0, 2, lambda a: ctl(H)), "swap": (0, 2, lambda a: SWAP),
    "crz": (1, 2, lambda a: ctl(R(a[0], Z))), "cu1": (1, 2, lambda a: ctl(U(0, 0, a[0]))),
    "cu3": (3, 2, lambda a: ctl(U(*a))),
    "rzz": (1, 2, lambda a: np.diag(np.exp(-1j * a[0] / 2 * np.array([1, -1, -1, 1])))),
    "rxx": (1, 2, lambda a: np.cos(a[0] / 2) * np.eye(4) - 1j * np.sin(a[0] / 2) * np.kron(X, X)),
    "ccx": (0, 3, lambda a: np.eye(8)[[0, 1, 2, 3, 4, 5, 7, 6]]),
    "cswap": (0, 3, lambda a: np.eye(8)[[0, 1, 2, 3, 4, 6, 5, 7]]),
}


def test_random_program_matches_oracle(ctx):
    import qpp_b200 as qb
    rng = np.random.default_rng(21)
    n = 6
    lines, ops = [HEAD + f"qreg q[{n}];"], []
    names = sorted(GATES)
    for _ in range(80):
        g = names[int(rng.integers(len(names)))]
        npar, nq, fm = GATES[g]
        a = [float(x) for x in rng.uniform(-3, 3, npar)]
        qs = [int(x) for x in rng.choice(n, nq, replace=False)]
        par = "(" + ", ".join(repr(x) for x in a) + ")" if npar else ""
        lines.append(f"{g}{par} " + ", ".join(f"q[{x}]" for x in qs) + ";")
        ops.append((fm(a), qs))
    c = qb.Circuit.from_qasm("\n".join(lines))
    e = qb.Engine(ctx, c).execute()
    got = e.get_state().numpy()
    x = np.zeros(2 ** n, dtype=complex)
    x[0] = 1
    for M, qs in ops:
        x = orc.apply(x, M, qs, [2] * n)
    assert np.max(np.abs(got - x)) < 1e-12


def test_reset_and_if_are_deterministic(ctx):
    import qpp_b200 as qb
    src = HEAD + """qreg q[2]; creg c[1];
    x q[0];
    measure q[0] -> c[0];
    if (c == 1) x q[1];
    if (c == 0) x q[1];
    reset q[0];
    """
    c = qb.Circuit.from_qasm(src)
    for kind in (qb.KET, qb.RHO):
        e = qb.Engine(ctx, c, kind).set_seed(3).execute()
        st = e.get_state().numpy()
        want = np.zeros(4)
        want[1] = 1  # |01>: q0 reset, q1 flipped once
        got = np.abs(st) if kind == qb.KET else np.abs(np.diag(st))
        assert np.max(np.abs(got - want)) < 1e-12
        assert e.get_dits()[0] == [1]
