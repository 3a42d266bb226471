"""The oracle's qpp::sample (instruments.hpp:856-940): std::discrete_distribution
draws over the full basis from std::mt19937(seed), reported per target digit."""
import numpy as np
import pytest

from oracle import oracle as orc


def test_sample_born_rule_and_digits():
    psi = np.array([0.6, 0, 0, 0.8j])
    d = orc.sample(psi, [1, 0], [2, 2], 20000, seed=4)
    assert set(map(tuple, d.tolist())) <= {(0, 0), (1, 1)}
    f = np.mean(d[:, 0] == 0)
    assert abs(f - 0.36) < 4 * np.sqrt(0.36 * 0.64 / 20000)


def test_sample_density_matrix_uses_the_diagonal():
    rho = np.diag([0.0, 0.25, 0.75, 0.0]).astype(np.complex128)
    d = orc.sample(rho, [0, 1], [2, 2], 4000, seed=1)
    assert set(map(tuple, d.tolist())) <= {(0, 1), (1, 0)}


def test_sample_is_reproducible_and_validates():
    psi = np.ones(8) / np.sqrt(8)
    a = orc.sample(psi, [2], [2, 2, 2], 50, seed=9)
    b = orc.sample(psi, [2], [2, 2, 2], 50, seed=9)
    assert np.array_equal(a, b)
    with pytest.raises(Exception):
        orc.sample(psi, [2], [2, 2, 2], 0)
    with pytest.raises(Exception):
        orc.sample(psi, [3], [2, 2, 2], 5)
