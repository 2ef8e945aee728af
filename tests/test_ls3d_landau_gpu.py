"""GPU parity of the 3D Landau LS solver (spectral_solver_landau_3d): against
the reference's own outputs (golden: fixed iteration counts, converged, smooth
capping) and against the oracle at 64^3, where the warp-line z-line kernel
with the law compiled in runs.  Tolerance 1e-9 relative."""
import numpy as np
import pytest

from mgkmc_b200 import workloads as W
from oracle import ls as OL

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def test_matches_reference(golden):
    from mgkmc_b200.linear_elastic_simulator import spectral_solver_landau_3d
    g = golden("ls3d_landau_12x8x6")
    v1, v2, v3, g1, g2, g3, g4 = g["v"]
    kw = dict(v1=v1, v2=v2, v3=v3, g1=g1, g2=g2, g3=g3, g4=g4, eps_bar=g["eps_bar"], eps_plastic=g["eps_plastic"])
    for k in (1, 3):
        eps, sig, _, _ = spectral_solver_landau_3d(g["lam"], g["mu"], **kw, max_iter=k, tol=0.0)
        assert rel(eps, g[f"eps_it{k}"]) < 1e-9 and rel(sig, g[f"sig_it{k}"]) < 1e-9
    eps, sig, _, _ = spectral_solver_landau_3d(g["lam"], g["mu"], **kw, max_iter=400, tol=1e-12)
    assert rel(eps, g["eps_conv"]) < 1e-9 and rel(sig, g["sig_conv"]) < 1e-9
    eps, sig, _, _ = spectral_solver_landau_3d(g["lam"], g["mu"], **kw, max_iter=400, tol=1e-12,
                                               strain_capping_enabled=True, strain_capping_limit=0.01,
                                               strain_capping_type="smooth", strain_capping_smooth_power=2.0)
    assert rel(eps, g["eps_cap"]) < 1e-9 and rel(sig, g["sig_cap"]) < 1e-9


@pytest.mark.parametrize("cap", [None, "piecewise"])
def test_warp_line_size_matches_oracle(golden, cap):
    from mgkmc_b200.linear_elastic_simulator import spectral_solver_landau_3d
    v = tuple(golden("ls3d_landau_12x8x6")["v"])
    n = 64
    rng = np.random.default_rng(64)
    E, nu = W.ls3d_material(n, n, n, rng)
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    ep = W.pure_shear_eigenstrain_3d(n, n, n, rng, frac=0.05)
    eb = np.array([[0.008, 0.001, 0.0], [0.001, -0.003, 0.0], [0.0, 0.0, -0.002]])
    o_eps, o_sig, _, _ = OL.spectral_solver_landau_3d(lam, mu, v, eb, ep, max_iter=200, tol=1e-10, cap_type=cap,
                                                      cap_limit=0.01)
    v1, v2, v3, g1, g2, g3, g4 = v
    eps, sig, _, _ = spectral_solver_landau_3d(lam, mu, v1, v2, v3, g1, g2, g3, g4, eb, ep, max_iter=200, tol=1e-10,
                                               strain_capping_enabled=cap is not None, strain_capping_limit=0.01,
                                               strain_capping_type=cap or "piecewise")
    assert rel(eps, o_eps) < 1e-9 and rel(sig, o_sig) < 1e-9
