"""The nonlinear load ramps (secant, Rose and Landau drivers,
linear_elastic_simulator.py:1353-2517) on the device solvers, against the
reference's own ramps (fixture nl_ramps) and the reference's Landau ramp test
(tests/test_landau_small_strain.py:131-160)."""
import numpy as np
import pytest

from mgkmc_b200 import linear_elastic_simulator as les
from test_nl_ramps_cpu import TAGS, _rel, run_ramp

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("tag", TAGS)
def test_ramp_on_device_matches_reference(golden, tag):
    # every solve stops at an update norm of 1e-11 and every macro loop at a
    # stress error of 1e3 Pa (1e-6 of the stresses); the device and the
    # reference reach the same iterates up to their solvers' rounding
    g = golden("nl_ramps")
    em, sm, el, sl = run_ramp(g, tag)
    assert em.shape == g[f"{tag}_eps_mac"].shape and len(el) == 4
    assert _rel(em, g[f"{tag}_eps_mac"]) < 1e-8
    assert _rel(sm, g[f"{tag}_sig_mac"]) < 1e-8
    assert _rel(el[-1], g[f"{tag}_eps"]) < 1e-8
    assert _rel(sl[-1], g[f"{tag}_sig"]) < 1e-8


def test_landau_simulation_2d_reference_case():
    # homogeneous 8x8, every component strain-controlled, five load steps:
    # the final macro strain is the target
    E, nu = 70.0e9, 0.3
    lam = np.full((8, 8), E * nu / ((1 + nu) * (1 - 2 * nu)))
    mu = np.full((8, 8), E / (2 * (1 + nu)))
    target = np.array([[0.02, 0.0], [0.0, -0.006]])
    em, sm, el, sl = les.landau_elastic_simulation_2d(
        lam, mu, -100.0e9, -50.0e9, -10.0e9, -1000.0e9, 500.0e9, -100.0e9, -200.0e9,
        np.ones((2, 2), dtype=bool), target, n_steps=5, pixel=1.0, plane_mode="plane_strain", store=True,
        enable_console=False)
    assert em.shape == (6, 2, 2) and sm.shape == (6, 2, 2) and len(el) == 6
    np.testing.assert_allclose(em[-1], target, atol=1e-7)
