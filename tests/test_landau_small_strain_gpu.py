"""The reference's Landau small-strain solver tests
(tests/test_landau_small_strain.py:10-128) run on the drop-ins: homogeneous
media, where the LS fixed point is the applied macro strain everywhere."""
import numpy as np
import pytest

from mgkmc_b200 import linear_elastic_simulator as les

pytestmark = pytest.mark.gpu

E, NU = 70.0e9, 0.3
V = dict(v1=-100.0e9, v2=-50.0e9, v3=-10.0e9, g1=-1000.0e9, g2=500.0e9, g3=-100.0e9, g4=-200.0e9)
LAM3 = E * NU / ((1 + NU) * (1 - 2 * NU))  # 3D (and 2D plane-strain) Lame lambda
MU = E / (2 * (1 + NU))


def test_landau_2d_plane_strain():
    lam, mu = np.full((16, 16), LAM3), np.full((16, 16), MU)
    eps_bar = np.array([[0.01, 0.002], [0.002, -0.005]])
    eps, sig, epsM, sigM = les.spectral_solver_landau_2d(lam=lam, mu=mu, **V, eps_bar=eps_bar, eps_plastic=None,
                                                         max_iter=100, tol=1e-8, verbose=True, pixel=1.0,
                                                         plane_mode="plane_strain")
    assert eps.shape == (16, 16, 2, 2) and sig.shape == (16, 16, 2, 2)
    np.testing.assert_allclose(epsM, eps_bar, atol=1e-7)
    np.testing.assert_allclose(eps[0, 0], eps_bar, atol=1e-7)


def test_landau_2d_plane_stress():
    lam, mu = np.full((16, 16), LAM3), np.full((16, 16), MU)
    eps_bar = np.array([[0.01, 0.0], [0.0, -0.003]])
    eps, sig, epsM, sigM = les.spectral_solver_landau_2d(lam=lam, mu=mu, **V, eps_bar=eps_bar, eps_plastic=None,
                                                         max_iter=100, tol=1e-8, verbose=True, pixel=1.0,
                                                         plane_mode="plane_stress")
    assert eps.shape == (16, 16, 2, 2) and sig.shape == (16, 16, 2, 2)
    np.testing.assert_allclose(epsM, eps_bar, atol=1e-7)


def test_landau_3d():
    lam, mu = np.full((8, 8, 8), LAM3), np.full((8, 8, 8), MU)
    eps_bar = np.array([[0.01, 0.002, 0.0], [0.002, -0.005, 0.001], [0.0, 0.001, 0.003]])
    eps, sig, epsM, sigM = les.spectral_solver_landau_3d(lam=lam, mu=mu, **V, eps_bar=eps_bar, eps_plastic=None,
                                                         max_iter=100, tol=1e-8, verbose=True, pixel=1.0)
    assert eps.shape == (8, 8, 8, 3, 3) and sig.shape == (8, 8, 8, 3, 3)
    np.testing.assert_allclose(epsM, eps_bar, atol=1e-7)
