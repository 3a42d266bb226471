"""OpenQASM 2.0 reader (qpp::qasm::read_from_string, qasm/qasm.hpp:781-820):
registers, broadcasting, gate definitions, measurement / reset / if steps
and the parse errors. Host-only: circuits are built without a GPU."""
import pytest

import qpp_b200 as qb

HEAD = 'OPENQASM 2.0;\ninclude "qelib1.inc";\n'


def steps(src):
    return qb.Circuit.from_qasm(HEAD + src).steps()


def test_registers_and_shape():
    c = qb.Circuit.from_qasm(HEAD + "qreg a[2]; qreg b[3]; creg m[4]; creg n[1];")
    assert (c.nq, c.d, c.nc, c.steps()) == (5, 2, 5, 0)


def test_broadcasting_and_builtins():
    assert steps("qreg q[3]; h q;") == 3
    assert steps("qreg q[2]; qreg r[2]; cx q, r;") == 2
    assert steps("qreg q[2]; qreg r[1]; cx q, r[0];") == 2
    assert steps("qreg q[3]; U(0.1, 0.2, 0.3) q[1]; CX q[0], q[2]; u2(0, pi) q[0];") == 3
    assert steps("qreg q[3]; ccx q[0], q[1], q[2]; rzz(pi/3) q[0], q[1];") == 2
    assert steps("qreg q[1]; rx(-pi/2 + 2*0.5^2) q[0]; rz(sqrt(2) * cos(pi)) q[0]; // comment\n") == 2


def test_gate_definitions_expand():
    src = """qreg q[3];
    gate bell a, b { h a; cx a, b; }
    gate rot(t) a { rz(t/2) a; barrier a; ry(-t) a; }
    bell q[0], q[1];
    rot(0.4) q;
    """
    assert steps(src) == 2 + 3 * 2


def test_measure_reset_and_if():
    src = """qreg q[2]; creg c[2];
    measure q -> c;
    reset q[1];
    if (c == 2) x q[0];
    """
    assert steps(src) == 2 + 1 + 3  # 2 measurements, 1 reset, IF + gate + END


@pytest.mark.parametrize("src,msg", [
    ("qreg q[2]; foo q[0];", "unknown gate"),
    ("qreg q[2]; rx q[0];", "wrong number"),
    ("qreg q[2]; h q[2];", "index out of range"),
    ("qreg q[2]; qreg r[3]; cx q, r;", "different sizes"),
    ("qreg q[1]; opaque g a;", "opaque"),
    ("qreg q[1]; creg c[1]; measure q[0] -> d[0];", "unknown creg"),
    ("qreg q[1]; rz(t) q[0];", "unknown parameter"),
])
def test_parse_errors(src, msg):
    with pytest.raises(qb.InvalidArgument) as e:
        qb.Circuit.from_qasm(HEAD + src)
    assert msg in str(e.value) and "line" in str(e.value)


def test_header_and_includes():
    with pytest.raises(qb.InvalidArgument):
        qb.Circuit.from_qasm("OPENQASM 3.0; qreg q[1];")
    with pytest.raises(qb.InvalidArgument):
        qb.Circuit.from_qasm('OPENQASM 2.0; include "other.inc"; qreg q[1];')


def test_qelib1_bodies_expand_as_qpp_does():
    """cu1, cu3 and cswap are not in qpp's table of known matrices, so qpp's
    reader expands their qelib1 bodies (qasmtools' standard library,
    qasmtools/include/qasmtools/parser/preprocessor.hpp:86-127): one step per
    U or known gate, which is where a noisy engine draws noise; r is one U."""
    assert steps("qreg q[2]; cu1(0.3) q[0], q[1];") == 5
    assert steps("qreg q[2]; cu3(0.1, 0.2, 0.3) q[0], q[1];") == 6
    assert steps("qreg q[3]; cswap q[2], q[0], q[1];") == 3
    assert steps("qreg q[1]; r(0.4, 0.7) q[0];") == 1
    assert steps("qreg a[2]; qreg b[2]; cu1(0.3) a, b;") == 10  # broadcast
