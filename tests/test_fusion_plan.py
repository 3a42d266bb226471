"""Host-side fusion planner (no GPU): pass counts and block structure."""
import qpp_b200 as qb


def test_layered_circuit_fuses_to_few_passes():
    c = qb.layered_circuit(30, 40, 1234)
    assert c.steps() == 1800
    p6 = c.fused_passes(6)
    p3 = c.fused_passes(3)
    # 15 pairs per layer, at most 3 pairs per 6-qubit block
    assert 150 <= p6 <= 240, p6
    assert p6 < p3 < 1800


def test_single_gates_are_one_pass_each_when_max_k_is_small():
    import numpy as np
    c = qb.Circuit(8)
    H = np.array([[1, 1], [1, -1]]) / np.sqrt(2)
    for q in range(8):
        c.gate(H, [q])
    assert c.fused_passes(1) == 8
    assert c.fused_passes(6) == 2  # two disjoint blocks of <= 6 qubits


def test_circuit_step_errors_follow_qcircuit():
    import numpy as np
    import pytest
    c = qb.Circuit(3)
    X = np.array([[0, 1], [1, 0]])
    with pytest.raises(qb.OutOfRange):
        c.gate(X, [3])
    with pytest.raises(qb.Duplicates):
        c.gate(np.kron(X, X), [1, 1])
    with pytest.raises(qb.MatrixMismatchSubsys):
        c.gate(X, [0, 1])
