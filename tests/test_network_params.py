"""Closed-form network and line helpers of ``extraction.py:236-317`` (CPU),
with the reference's own tests (``tests/test_quasistatic.py``) as the model."""

import numpy as np
import pytest


def test_s_parameters_of_matched_load_are_zero():
    from fieldspice_b200 import extraction as EX
    S = EX.s_parameters(np.diag([1 / 50.0, 1 / 50.0]), 50.0)
    assert np.abs(S).max() < 1e-12


def test_s_parameters_are_passive_and_reciprocal():
    from fieldspice_b200 import extraction as EX
    Y = np.array([[1 / 50 + 1e-6, -1e-6], [-1e-6, 1 / 50 + 1e-6]])
    S = EX.s_parameters(Y, 50.0)
    assert np.linalg.svd(S, compute_uv=False).max() <= 1.0 + 1e-12
    assert np.allclose(S, S.T)
    stack = EX.s_parameters(np.stack([Y, 2 * Y]), np.array([50.0, 75.0]))
    assert stack.shape == (2, 2, 2)


def test_y_z_round_trip():
    from fieldspice_b200 import extraction as EX
    Y = np.array([[3.0, -1.0], [-1.0, 2.0]])
    assert np.allclose(EX.z_to_y(EX.y_to_z(Y)), Y)


def test_skin_depth_and_elmore():
    from fieldspice_b200 import extraction as EX
    assert EX.skin_depth(5.8e7, 1e9) == pytest.approx(2.09e-6, rel=5e-3)
    assert EX.skin_depth(5.8e7, 0.0) == float("inf")
    assert EX.elmore_delay([1.0, 2.0], [3.0, 4.0]) == pytest.approx(3 * 1 + 4 * 3)
    with pytest.raises(ValueError):
        EX.elmore_delay([1.0], [1.0, 2.0])


def test_characteristic_impedance_and_lc_identity():
    from fieldspice_b200 import extraction as EX
    from fieldspice_b200.units import eps0, mu0
    C = np.array([[1e-10]])
    L = mu0 * eps0 / C
    r = {"R": np.zeros((1, 1)), "L": L, "G": np.zeros((1, 1)), "C": C}
    assert EX.check_lc_identity(r) < 1e-14
    z_dc = EX.characteristic_impedance(r)
    z_hf = EX.characteristic_impedance(r, 1e9)
    assert np.allclose(z_hf.real, z_dc) and np.abs(z_hf.imag).max() < 1e-9
