"""qpp's noise models (include/qpp/classes/noise.hpp:388-597) as Kraus sets
for Engine.set_noise.

Each model is (Ks, probs): probs is a list for a state-independent model
(NoiseType::StateIndependent, one Kraus index drawn from probs) and None for
a state-dependent one (p_i = tr(K_i rho_q K_i^dagger) of the qudit's reduced
state, noise.hpp:100-121). Two of qpp's conventions are kept on purpose, so
that an engine given these models draws what qpp draws:

* QubitAmplitudeDampingNoise(gamma) uses K0 = [[1, 0], [0, sqrt(gamma)]],
  K1 = [[0, sqrt(1 - gamma)], [0, 0]] (noise.hpp:493-496): gamma is the
  amplitude that survives, not the decay probability;
* QuditDepolarizingNoise(p, D) gives every non-identity Weyl operator the
  weight p (noise.hpp:566-575: p / (D - 1) * (D - 1)), so after
  std::discrete_distribution's normalisation the identity has probability
  (1 - p) / (1 + (D^2 - 2) p).
"""
from __future__ import annotations

import numpy as np


class NoiseModel:
    """Kraus operators of one qudit and, when state-independent, their
    probabilities."""

    def __init__(self, name, Ks, probs=None):
        self.name = name
        self.Ks = [np.asarray(K, dtype=np.complex128) for K in Ks]
        self.probs = None if probs is None else [float(x) for x in probs]

    @property
    def d(self):
        return self.Ks[0].shape[0]

    @property
    def state_dependent(self):
        return self.probs is None


def _out_of_range(where, what):
    from . import OutOfRange
    return OutOfRange(12, where, what)


def _check(x, name, cls):
    if x < 0 or x > 1:
        raise _out_of_range(f"qpp::{cls}::{cls}()", name)


_I = np.eye(2, dtype=np.complex128)
_X = np.array([[0, 1], [1, 0]], dtype=np.complex128)
_Y = np.array([[0, -1j], [1j, 0]], dtype=np.complex128)
_Z = np.array([[1, 0], [0, -1]], dtype=np.complex128)


def QubitDepolarizingNoise(p):
    """{I, X, Y, Z} with {1 - p, p/3, p/3, p/3} (noise.hpp:388-408)."""
    _check(p, "p", "QubitDepolarizingNoise")
    return NoiseModel("QubitDepolarizingNoise", [_I, _X, _Y, _Z], [1 - p, p / 3, p / 3, p / 3])


def QubitPhaseFlipNoise(p):
    """{I, Z} with {1 - p, p} (noise.hpp:414-432)."""
    _check(p, "p", "QubitPhaseFlipNoise")
    return NoiseModel("QubitPhaseFlipNoise", [_I, _Z], [1 - p, p])


def QubitBitFlipNoise(p):
    """{I, X} with {1 - p, p} (noise.hpp:438-456)."""
    _check(p, "p", "QubitBitFlipNoise")
    return NoiseModel("QubitBitFlipNoise", [_I, _X], [1 - p, p])


def QubitBitPhaseFlipNoise(p):
    """{I, Y} with {1 - p, p} (noise.hpp:462-480)."""
    _check(p, "p", "QubitBitPhaseFlipNoise")
    return NoiseModel("QubitBitPhaseFlipNoise", [_I, _Y], [1 - p, p])


def QubitAmplitudeDampingNoise(gamma):
    """State-dependent; qpp's convention (noise.hpp:486-505)."""
    _check(gamma, "gamma", "QubitAmplitudeDampingNoise")
    K0 = np.array([[1, 0], [0, np.sqrt(gamma)]], dtype=np.complex128)
    K1 = np.array([[0, np.sqrt(1 - gamma)], [0, 0]], dtype=np.complex128)
    return NoiseModel("QubitAmplitudeDampingNoise", [K0, K1])


def QubitPhaseDampingNoise(lam):
    """State-dependent (noise.hpp:511-530)."""
    _check(lam, "lambda", "QubitPhaseDampingNoise")
    K0 = np.array([[1, 0], [0, np.sqrt(1 - lam)]], dtype=np.complex128)
    K1 = np.array([[0, 0], [0, np.sqrt(lam)]], dtype=np.complex128)
    return NoiseModel("QubitPhaseDampingNoise", [K0, K1])


def QuditDepolarizingNoise(p, D):
    """Xd^i Zd^j for i, j in [0, D) (row-major in (i, j)), probabilities
    {1 - p, p, ..., p} (noise.hpp:538-597)."""
    if D < 2:
        raise _out_of_range("qpp::QuditDepolarizingNoise::QuditDepolarizingNoise()", "D")
    _check(p, "p", "QuditDepolarizingNoise")
    w = np.exp(2j * np.pi / D)
    Xd = np.zeros((D, D), dtype=np.complex128)
    for j in range(D):
        Xd[(j + 1) % D, j] = 1
    Zd = np.diag([w ** j for j in range(D)])
    Ks = [np.linalg.matrix_power(Xd, i) @ np.linalg.matrix_power(Zd, j)
          for i in range(D) for j in range(D)]
    probs = [1 - p] + [p / (D - 1) * (D - 1)] * (D * D - 1)
    return NoiseModel("QuditDepolarizingNoise", Ks, probs)
