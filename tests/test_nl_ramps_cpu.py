"""Host logic of the nonlinear load ramps (the secant, Rose and Landau
drivers of linear_elastic_simulator.py:1353-2517): the drop-in ramps run here
with the oracle's solvers put in place of the device solvers, and are
compared with the reference's own ramps (fixture nl_ramps, made by
tests/golden/make_golden.py).  The device solvers are pinned by their own
tests; tests/test_nl_ramps_gpu.py runs the ramps on them."""
import os

import numpy as np
import pytest

from mgkmc_b200 import linear_elastic_simulator as les
from oracle import ls as OL


def _rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / np.max(np.abs(b)))


@pytest.fixture
def oracle_solvers(monkeypatch):
    def sec2(lam, mu, d, k, eps_bar, max_iter=400, tol=1e-6, pixel=1.0, plane_mode="plane_strain", eps_init=None):
        assert plane_mode == "plane_strain"
        return OL.spectral_solver_secant_2d(lam, mu, d, k, eps_bar, max_iter=max_iter, tol=tol, pixel=pixel,
                                            eps_init=eps_init)

    def sec3(lam, mu, d, k, eps_bar, max_iter=400, tol=1e-6, pixel=1.0, eps_init=None):
        return OL.spectral_solver_secant_3d(lam, mu, d, k, eps_bar, max_iter=max_iter, tol=tol, pixel=pixel,
                                            eps_init=eps_init)

    def rose(lam, mu, eta, floor_f, eps_bar=None, max_iter=400, tol=1e-6, pixel=1.0, plane_mode="plane_strain",
             eps_init=None):
        return OL.spectral_solver_rose_2d(lam, mu, eta, floor_f, eps_bar, max_iter=max_iter, tol=tol, pixel=pixel,
                                          plane_mode=plane_mode, eps_init=eps_init)

    def lan2(lam, mu, v1, v2, v3, g1, g2, g3, g4, eps_bar, max_iter=400, tol=1e-6, pixel=1.0,
             plane_mode="plane_strain", eps_init=None, e33_state=None, solver="dbfft", strain_capping_enabled=False,
             **cap):
        assert plane_mode == "plane_strain" and solver == "dbfft" and not strain_capping_enabled
        return OL.spectral_solver_landau_2d(lam, mu, (v1, v2, v3, g1, g2, g3, g4), eps_bar, max_iter=max_iter, tol=tol,
                                            pixel=pixel, eps_init=eps_init)

    def lan3(lam, mu, v1, v2, v3, g1, g2, g3, g4, eps_bar, max_iter=400, tol=1e-6, pixel=1.0, eps_init=None,
             solver="dbfft", strain_capping_enabled=False, **cap):
        assert solver == "dbfft" and not strain_capping_enabled
        return OL.spectral_solver_landau_3d(lam, mu, (v1, v2, v3, g1, g2, g3, g4), eps_bar, max_iter=max_iter, tol=tol,
                                            pixel=pixel, eps_init=eps_init)

    for name, fn in (("spectral_solver_secant_2d", sec2), ("spectral_solver_secant_3d", sec3),
                     ("spectral_solver_rose_2d", rose), ("spectral_solver_landau_2d", lan2),
                     ("spectral_solver_landau_3d", lan3)):
        monkeypatch.setattr(les, name, fn)


COMMON = dict(n_steps=3, tol_ls=1e-11, max_iter_ls=600, tol_macro=1e3, max_iter_macro=30, store=True,
              enable_console=False)


def run_ramp(g, tag, **kw):
    v = tuple(g["v"])
    if tag.endswith("3d"):
        lam, mu, m = g["lam3"], g["mu3"], g["mask3"]
    else:
        lam, mu, m = g["lam2"], g["mu2"], g["mask2"]
    t = g[f"{tag}_target"]
    args = dict(COMMON, **kw)
    if tag == "secant2d":
        return les.secant_elastic_simulation_2d(lam, mu, 0.3, 50.0, m, t, **args)
    if tag == "rose2d":
        return les.rose_elastic_simulation_2d(lam, mu, 30.0, 0.1, m, t, **args)
    if tag == "rose2d_pst":
        return les.rose_elastic_simulation_2d(lam, mu, 30.0, 0.1, m, t, plane_mode="plane_stress", **args)
    if tag == "secant3d":
        return les.secant_elastic_simulation_3d(lam, mu, 0.3, 50.0, m, t, **args)
    if tag == "landau2d":
        return les.landau_elastic_simulation_2d(lam, mu, *v, m, t, **args)
    return les.landau_elastic_simulation_3d(lam, mu, *v, m, t, **args)


TAGS = ("secant2d", "rose2d", "rose2d_pst", "secant3d", "landau2d", "landau3d")


@pytest.mark.parametrize("tag", TAGS)
def test_ramp_matches_reference(golden, oracle_solvers, tag):
    g = golden("nl_ramps")
    em, sm, el, sl = run_ramp(g, tag)
    assert em.shape == g[f"{tag}_eps_mac"].shape and len(el) == 4
    assert _rel(em, g[f"{tag}_eps_mac"]) < 1e-9
    assert _rel(sm, g[f"{tag}_sig_mac"]) < 1e-9
    assert _rel(el[-1], g[f"{tag}_eps"]) < 1e-9
    assert _rel(sl[-1], g[f"{tag}_sig"]) < 1e-9


def test_ramp_outputs(golden, oracle_solvers, tmp_path):
    # logs in the reference's layout, VTK files on the "last" schedule with
    # the secant moduli, checkpoints every step (the reference passes no
    # moduli there and cannot write them; here the linear ones)
    from mgkmc_b200 import checkpoint as C
    from mgkmc_b200.vtk import read_vtu
    g = golden("nl_ramps")
    log, glog = tmp_path / "ramp.log", tmp_path / "global.log"
    vtk, chk = str(tmp_path / "v"), str(tmp_path / "c" / "chk")
    em, sm, el, sl = run_ramp(g, "secant2d", log_path=str(log), global_log_path=str(glog), vtk_path=vtk,
                              vtk_interval="last", checkpoint_interval=1, checkpoint_path=chk)
    lines = log.read_text().splitlines()
    assert lines[0].split() == ["Timestamp", "Elapsed(s)", "Step", "Eps_xx", "Sig_xx(GPa)"]
    assert len([ln for ln in lines[2:] if ln and ln[0].isdigit()]) == 4
    assert "Total Duration" in log.read_text()
    rows = [ln.split() for ln in glog.read_text().splitlines()[2:]]
    assert [r[0] for r in rows] == ["0", "1", "2", "3"] and len(rows[0]) == 7
    np.testing.assert_allclose(float(rows[3][1]), em[3][0, 0], atol=1e-6)
    assert sorted(os.listdir(tmp_path)) == ["c", "global.log", "ramp.log", "v_final.vtu"]
    _, _, pd, cd = read_vtu(vtk + "_final.vtu")
    lam, mu = g["lam2"], g["mu2"]
    mu_sec = mu * (1.0 - 0.3 * (1.0 - np.exp(-50.0 * les._vm_eq_2d(el[-1]))))
    np.testing.assert_allclose(cd["E"], (mu_sec * (3 * lam + 2 * mu_sec) / (lam + mu_sec)).ravel(), rtol=1e-12)
    assert len(os.listdir(tmp_path / "c")) == 4
    data, attrs = C.load(chk + "_000003")
    np.testing.assert_array_equal(data["fields/eps_field"], el[-1])
    assert attrs["metadata"]["step"] == 3


def test_landau_3d_global_log_has_every_component(golden, oracle_solvers, tmp_path):
    g = golden("nl_ramps")
    glog = tmp_path / "g.log"
    em, sm, _, _ = run_ramp(g, "landau3d", global_log_path=str(glog), store=False)
    hdr = glog.read_text().splitlines()[0].split()
    rows = [ln.split() for ln in glog.read_text().splitlines()[2:]]
    assert len(hdr) == 13 and all(len(r) == 13 for r in rows)
    np.testing.assert_allclose([float(x) for x in rows[-1][1:7]],
                               [em[-1][c] for c in ((0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2))], atol=1e-6)


def test_vm_equivalent_strains():
    # the equivalent strains of the VTK moduli against direct evaluations of
    # sqrt(2/3 e':e') (plane strain: e33 = 0 enters the deviator)
    rng = np.random.default_rng(5)
    e2 = rng.normal(0, 0.01, (4, 3, 2, 2))
    full = np.zeros((4, 3, 3, 3))
    full[..., :2, :2] = 0.5 * (e2 + np.swapaxes(e2, -1, -2))
    dev = full - np.trace(full, axis1=-2, axis2=-1)[..., None, None] * np.eye(3) / 3
    np.testing.assert_allclose(les._vm_eq_2d(e2), np.sqrt(2 / 3 * np.sum(dev ** 2, axis=(-2, -1))), rtol=1e-13)
    e3 = rng.normal(0, 0.01, (2, 3, 4, 3, 3))
    s3 = 0.5 * (e3 + np.swapaxes(e3, -1, -2))
    d3 = s3 - np.trace(s3, axis1=-2, axis2=-1)[..., None, None] * np.eye(3) / 3
    np.testing.assert_allclose(les._vm_eq_3d(e3), np.sqrt(2 / 3 * np.sum(d3 ** 2, axis=(-2, -1))), rtol=1e-13)


@pytest.mark.parametrize("tag", TAGS)
def test_ramp_vtk_moduli_match_reference(golden, oracle_solvers, monkeypatch, tmp_path, tag):
    # the (E, nu) fields written with the final VTK file: the secant and Rose
    # ramps' secant moduli of the final strain (Rose plane stress with its
    # e33 fixed point), the Landau ramps' linear moduli
    from mgkmc_b200 import vtk
    seen = {}

    def record(fname, eps, sig, E, nu, pixel=1.0, **kw):
        seen["name"], seen["E"], seen["nu"] = fname, np.array(E), np.array(nu)

    monkeypatch.setattr(vtk, "export_to_vtk", record)
    g = golden("nl_ramps")
    run_ramp(g, tag, vtk_path=str(tmp_path / "r"), vtk_interval="last", store=False)
    assert seen["name"] == str(tmp_path / "r") + "_final.vtu"
    np.testing.assert_allclose(seen["E"], g[f"{tag}_vtk_E"], rtol=1e-12)
    np.testing.assert_allclose(seen["nu"], g[f"{tag}_vtk_nu"], rtol=1e-12)
