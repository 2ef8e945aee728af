"""Without a CUDA device the public drop-ins raise instead of computing on the
host: the product path has no CPU fallback (the numpy restatement under
oracle/ is test infrastructure and is never reached from mgkmc_b200)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.skipif(torch.cuda.is_available(), reason="checks the device-less behaviour")

NO_FALLBACK = "no CPU fallback"


def test_small_strain_solvers_raise():
    from mgkmc_b200 import linear_elastic_simulator as les
    E, nu = np.full((8, 8), 1e11), np.full((8, 8), 0.3)
    with pytest.raises(RuntimeError, match=NO_FALLBACK):
        les.spectral_solver_2d(E, nu, np.zeros((2, 2)))
    with pytest.raises(RuntimeError, match=NO_FALLBACK):
        les.spectral_solver_3d(np.full((4, 4, 4), 1e11), np.full((4, 4, 4), 0.3), np.zeros((3, 3)))
    with pytest.raises(RuntimeError, match=NO_FALLBACK):
        les.Ls2dBatch([(8, 8)])


def test_finite_strain_step_raises():
    from mgkmc_b200 import finite_strain_simulator as fss
    n = 4
    F = np.broadcast_to(np.eye(3)[:, :, None, None, None], (3, 3, n, n, n)).copy()
    with pytest.raises(RuntimeError, match=NO_FALLBACK):
        fss.finite_strain_solver_step_3d(F, np.eye(3), solver="newton_cg", model_type="svk",
                                         lam=np.full((n, n, n), 5e10), mu=np.full((n, n, n), 3e10))


def test_kmc_dropins_raise():
    from mgkmc_b200 import kmc_simulator_functions as kf
    from mgkmc_b200 import stz
    Q = np.ones((4, 4, 2))
    with pytest.raises(RuntimeError, match=NO_FALLBACK):
        kf.compute_rates_2d(Q, 1e-28, 300.0)
    with pytest.raises(RuntimeError, match=NO_FALLBACK):
        stz.compute_rates(np.ones((4, 4, 4, 2)), 1e-28, 300.0)


def test_server_raises():
    from mgkmc_b200.serving import Server
    with pytest.raises(RuntimeError, match=NO_FALLBACK):
        Server()
