"""qpp's noise models (noise.hpp:388-597) as Kraus sets, conventions kept."""
import numpy as np
import pytest

import qpp_b200 as qb
from qpp_b200 import noise


@pytest.mark.parametrize("make", [noise.QubitDepolarizingNoise, noise.QubitPhaseFlipNoise,
                                  noise.QubitBitFlipNoise, noise.QubitBitPhaseFlipNoise])
def test_pauli_models_are_unitary_mixtures(make):
    m = make(0.1)
    assert not m.state_dependent and abs(sum(m.probs) - 1) < 1e-15 and m.probs[0] == 0.9
    for K in m.Ks:
        assert np.allclose(K.conj().T @ K, np.eye(2))


def test_damping_models_follow_qpp_conventions():
    ad = noise.QubitAmplitudeDampingNoise(0.3)
    assert ad.state_dependent
    assert np.allclose(ad.Ks[0], [[1, 0], [0, np.sqrt(0.3)]])      # noise.hpp:495
    assert np.allclose(ad.Ks[1], [[0, np.sqrt(0.7)], [0, 0]])      # noise.hpp:496
    pd = noise.QubitPhaseDampingNoise(0.2)
    s = sum(K.conj().T @ K for K in pd.Ks)
    assert np.allclose(s, np.eye(2))


def test_qudit_depolarizing_weights_and_operators():
    m = noise.QuditDepolarizingNoise(0.05, 3)
    assert len(m.Ks) == 9 and m.probs[0] == 0.95 and all(abs(p - 0.05) < 1e-15 for p in m.probs[1:])
    assert np.allclose(m.Ks[0], np.eye(3))
    w = np.exp(2j * np.pi / 3)
    assert np.allclose(m.Ks[1], np.diag([1, w, w * w]))             # Xd^0 Zd^1
    for K in m.Ks:
        assert np.allclose(K.conj().T @ K, np.eye(3))


def test_out_of_range():
    with pytest.raises(qb.OutOfRange):
        noise.QubitDepolarizingNoise(1.5)
    with pytest.raises(qb.OutOfRange):
        noise.QuditDepolarizingNoise(0.1, 1)
