"""GPU parity of the drivers around the solvers and of the solvers at the
sizes the benchmark runs:

* the mixed-BC load ramps ``linear_elastic_simulation_2d/3d`` and
  ``finite_strain_simulation_3d`` against the reference's own outputs
  (goldens made by running the unmodified reference), 1e-9 relative;
* the device-resident KMC driver against the reference's own trajectory
  (KmcSimulation2D.run_simulation with its RandomState draws): identical
  events, times and macro strain to 1e-9, fields 1e-9;
* the KMC driver at the benchmark's 256^2 x 8 grid (Q0 ~ N(1.0, 0.15) eV)
  against the oracle driver, 60 events from a pre-strained state;
* the finite-strain step at 64^3 (mixed BC) and 96^3 (Newton at a prescribed
  F_bar), where the warp-line passes run, against oracle fixtures, 1e-9;
* a checkpointed and resumed trajectory equal to an uninterrupted one, bit
  for bit.
"""
import numpy as np
import pytest

from mgkmc_b200 import workloads as W

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def test_linear_elastic_simulation_2d_matches_reference(golden):
    from mgkmc_b200.linear_elastic_simulator import linear_elastic_simulation_2d
    g = golden("ls2d_macro_16")
    epsM, sigM, eps_l, sig_l = linear_elastic_simulation_2d(
        g["E"], g["nu"], g["mask"], g["target"], n_steps=2, tol_ls=1e-10, max_iter_ls=300, tol_macro=1e3,
        max_iter_macro=30, enable_console=False)
    scale = np.max(np.abs(g["sigM"]))
    assert np.max(np.abs(sigM - g["sigM"])) < 1e-9 * scale
    assert np.max(np.abs(epsM - g["epsM"])) < 1e-9 * np.max(np.abs(g["epsM"]))
    assert rel(eps_l[-1], g["eps_last"]) < 1e-9
    assert rel(sig_l[-1], g["sig_last"]) < 1e-9


def test_ramps_write_vtk_on_the_reference_schedule(golden, tmp_path):
    # vtk_interval 2 over 3 load steps: files at steps 0 and 2 and the final
    # one (3 % 2 != 0), holding the step's fields (linear_elastic_simulator.py
    # :237-256); the finite-strain ramp with "last" writes only the final one
    from mgkmc_b200 import vtk as V
    from mgkmc_b200.finite_strain_simulator import finite_strain_simulation_2d
    from mgkmc_b200.linear_elastic_simulator import linear_elastic_simulation_2d
    g = golden("ls2d_macro_16")
    path = str(tmp_path / "ls")
    epsM, sigM, eps_l, sig_l = linear_elastic_simulation_2d(
        g["E"], g["nu"], g["mask"], g["target"], n_steps=3, tol_ls=1e-10, max_iter_ls=300, tol_macro=1e3,
        max_iter_macro=30, enable_console=False, vtk_path=path, vtk_interval=2)
    import os
    assert sorted(f for f in os.listdir(tmp_path) if f.endswith(".vtu")) == \
        ["ls_000000.vtu", "ls_000002.vtu", "ls_final.vtu"]
    _, _, _, cd = V.read_vtu(path + "_final.vtu")
    np.testing.assert_array_equal(cd["sig_xx"], sig_l[-1][..., 0, 0].ravel())
    np.testing.assert_array_equal(cd["eps_xy"], eps_l[-1][..., 0, 1].ravel())
    fpath = str(tmp_path / "fs")
    F_m, S_m, P_m, F_l, S_l = finite_strain_simulation_2d(
        g["E"], g["nu"], (0, 0), 0.004, 2, mixed_targets={}, tol_NW=1e-10, tol_CG=1e-11, max_NW=30,
        enable_console=False, model_type="svk", solver="newton_cg", vtk_path=fpath, vtk_interval="last")
    _, _, _, cd = V.read_vtu(fpath + "_final.vtu")
    np.testing.assert_array_equal(cd["sig_yy"], S_l[-1][1, 1].ravel())
    E_GL = 0.5 * (np.einsum("kixy,kjxy->ijxy", F_l[-1], F_l[-1]) - np.eye(2)[:, :, None, None])
    np.testing.assert_allclose(cd["eps_xx"], E_GL[0, 0].ravel(), rtol=0, atol=1e-15)


def test_linear_elastic_simulation_3d_matches_reference(golden):
    from mgkmc_b200.linear_elastic_simulator import linear_elastic_simulation_3d
    g = golden("ls3d_macro_8x6x4")
    epsM, sigM, eps_l, sig_l = linear_elastic_simulation_3d(
        g["E"], g["nu"], g["mask"], g["target"], n_steps=2, tol_ls=1e-10, max_iter_ls=300, tol_macro=1e3,
        max_iter_macro=30, enable_console=False)
    assert np.max(np.abs(sigM - g["sigM"])) < 1e-9 * np.max(np.abs(g["sigM"]))
    assert np.max(np.abs(epsM - g["epsM"])) < 1e-9 * np.max(np.abs(g["epsM"]))
    assert rel(eps_l[-1], g["eps_last"]) < 1e-9
    assert rel(sig_l[-1], g["sig_last"]) < 1e-9


def test_finite_strain_simulation_3d_matches_reference(golden):
    from mgkmc_b200.finite_strain_simulator import finite_strain_simulation_3d
    g = golden("fs3d_sim_6")
    Fm, Sm, Pm, F_l, S_l = finite_strain_simulation_3d(
        g["E"], g["nu"], (0, 0), 0.01, 2, mixed_targets={(1, 1): 0.0, (2, 2): 0.0}, tol_NW=1e-10, tol_CG=1e-11,
        max_NW=30, tol_macro=1e3, max_iter_macro=30, enable_console=False, model_type="svk", solver="newton_cg")
    assert np.max(np.abs(Fm - g["F_macro"])) < 1e-9
    assert np.max(np.abs(Pm - g["P_macro"])) < 1e-9 * np.max(np.abs(g["P_macro"]))
    assert np.max(np.abs(Sm - g["Sig_macro"])) < 1e-9 * np.max(np.abs(g["Sig_macro"]))
    assert rel(F_l[-1], g["F_last"]) < 1e-9
    assert rel(S_l[-1], g["Sig_last"]) < 1e-9


def _ref_draws(g):
    from mgkmc_b200.kmc import ReferenceDraws
    rs = np.random.RandomState()
    rs.set_state(("MT19937", g["rs_keys"], int(g["rs_pos"]), int(g["rs_has_gauss"]), float(g["rs_gauss"])))
    return ReferenceDraws(rs, 0.1, 0.6, 0.15, 0.3)


def test_kmc_driver_matches_reference_trajectory(golden):
    from mgkmc_b200.kmc import Kmc2D
    g = golden("kmc2d_traj_12x8")
    k = Kmc2D(g["E"], g["nu"], g["catalog0"], g["Q00"], T=300.0, strain_rate=1e7, step_size=float(g["step_size"]),
              jp=0.0, jt=0.0, cap=2.0, mixed_tol=1e4, mixed_max_iter=50, ls_tol=1e-6, ls_max_iter=200)
    r = k.run(_ref_draws(g), int(g["n_steps"]))
    assert len(r["events"]) == len(g["events"])
    np.testing.assert_array_equal(np.array([e[:3] for e in r["events"]]), g["events"])
    t = np.array([e[3] for e in r["events"]])
    assert np.max(np.abs(t - g["times"]) / np.abs(g["times"])) < 1e-9
    np.testing.assert_allclose(r["eps_macro"], g["eps_macro"], rtol=1e-9, atol=1e-15)
    assert rel(r["sig"], g["sig"]) < 1e-9
    np.testing.assert_array_equal(r["eps_p"], g["eps_plastic"])


def test_kmc_driver_at_benchmark_grid_matches_oracle():
    # 256^2 x 8 modes, Q0 ~ N(1.0, 0.15) eV clipped at 0.3 (the KMC
    # benchmark's grid and barriers), exact selection, cold FP64 LS at 1e-6;
    # started at 2.4 % strain, where the benchmark's events happen
    from mgkmc_b200.kmc import Kmc2D
    from oracle import kmc_driver as OD
    n, M = 256, 8
    rng0 = np.random.default_rng(1)
    E, nu = W.ls2d_material(n, n, rng0)
    cat, Q0 = W.kmc2d_state(n, n, M, rng0)
    e0 = np.array([[0.024, 0.0], [0.0, -0.42 * 0.024]])
    o = OD.run_kmc2d(E, nu, cat, Q0, np.random.default_rng(9), n_steps=40, max_events=60, eps_macro0=e0)
    k = Kmc2D(E, nu, cat, Q0)
    k.eps_macro = e0.copy()
    r = k.run(np.random.default_rng(9), 40, max_events=60)
    assert len(r["events"]) == len(o["events"]) == 60
    for (x, y, m, t), (xo, yo, mo, to) in zip(r["events"], o["events"]):
        assert (x, y, m) == (xo, yo, mo)
        assert abs(t - to) <= 1e-9 * abs(to)
    np.testing.assert_allclose(r["eps_macro"], o["eps_macro"], rtol=1e-9, atol=1e-15)
    assert rel(r["sig"], o["sig"]) < 1e-9
    np.testing.assert_array_equal(r["eps_p"], o["eps_p"])
    assert r["solves"] == o["solves"]


def _fs_compare(g, F, P, Fbo):
    Fs = np.moveaxis(F, (0, 1), (-2, -1)).reshape(-1, 9)
    Ps = np.moveaxis(P, (0, 1), (-2, -1)).reshape(-1, 9)
    idx = g["idx"]
    assert np.max(np.abs(Fs[idx] - g["F_s"])) < 1e-9 * g["F_max"]
    assert np.max(np.abs(Ps[idx] - g["P_s"])) < 1e-9 * g["P_max"]
    assert np.max(np.abs(Fs.mean(axis=0) - g["F_mean"])) < 1e-9 * g["F_max"]
    assert np.max(np.abs(Ps.mean(axis=0) - g["P_mean"])) < 1e-9 * g["P_max"]
    assert abs(np.linalg.norm(Fs - np.eye(3).ravel()) - g["F_norm"]) < 1e-9 * g["F_norm"]
    assert abs(np.linalg.norm(Ps) - g["P_norm"]) < 1e-9 * g["P_norm"]
    assert np.max(np.abs(Fbo - g["F_bar_out"])) < 1e-9


@pytest.mark.parametrize("n", [64, 96])
def test_finite_strain_warp_line_sizes_match_oracle(golden, n):
    # fixtures: tests/golden/make_oracle_large.py (the oracle at these sides)
    from mgkmc_b200.finite_strain_simulator import finite_strain_solver_step_3d
    g = golden(f"fs3d_neohookean_{n}_oracle")
    E, nu, Fp = W.fs3d_material(n, n, n, np.random.default_rng(n))
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    F0 = np.einsum("ij,xyz->ijxyz", np.eye(3), np.ones((n, n, n)))
    if n == 64:
        Pm, Pt = g["P_mask"], np.zeros((3, 3))
    else:
        Pm = Pt = None
    F, P, Sig, _, Fb = finite_strain_solver_step_3d(
        F0, g["F_bar_in"], Fp=Fp, driving_component=(0, 0), P_target=Pt, P_mask=Pm, E_avg=E.mean(),
        nu_avg=nu.mean(), tol_NW=1e-10, tol_CG=1e-11, max_NW=40, tol_macro=1e3, max_iter_macro=40,
        enable_console=False, model_type="neo_hookean", solver="newton_cg", lam=lam, mu=mu)
    _fs_compare(g, F, P, Fb)


@pytest.mark.parametrize("selection,ls_start,precision", [("exact", "cold", "fp64"), ("fast", "warm", "mixed")])
def test_checkpoint_resume_is_bit_exact(tmp_path, selection, ls_start, precision):
    from mgkmc_b200 import checkpoint as C
    from mgkmc_b200.kmc import Kmc2D
    n, M = 32, 8
    rng0 = np.random.default_rng(5)
    E, nu = W.ls2d_material(n, n, rng0)
    cat, Q0 = W.kmc2d_state(n, n, M, rng0, q_mean=0.6)
    kw = dict(step_size=1e-4, strain_rate=1e7, q_mean=0.6, selection=selection, ls_start=ls_start,
              precision=precision)
    full = Kmc2D(E, nu, cat, Q0, **kw).run(np.random.default_rng(11), 60)
    a = Kmc2D(E, nu, cat, Q0, **kw)
    rng = np.random.default_rng(11)
    a.run(rng, 35)
    path = C.save_trajectory(str(tmp_path / "traj"), a, rng)
    st, rng2, meta = C.load_trajectory(path)
    assert meta["step"] == 35
    b = Kmc2D(st["E"], st["nu"], st["catalog"], st["Q0"], **kw)
    b.load_state_dict(st)
    res = b.run(rng2, 60)
    assert len(full["events"]) > 0
    assert res["events"] == full["events"]
    np.testing.assert_array_equal(res["sig"], full["sig"])
    np.testing.assert_array_equal(res["eps_p"], full["eps_p"])
    np.testing.assert_array_equal(res["eps_macro"], full["eps_macro"])
    assert res["time"] == full["time"] and res["solves"] == full["solves"]


@pytest.mark.parametrize("n,selection,ls_start,precision", [(32, "exact", "cold", "fp64"),
                                                           (64, "fast", "warm", "mixed")])
def test_kmc3d_checkpoint_resume_is_bit_exact(tmp_path, n, selection, ls_start, precision):
    # a 3D trajectory checkpointed after 20 AQS steps (the reference's 3D
    # layout plus the resume group) and resumed equals the uninterrupted run
    # (the mixed 3D form runs sides 64, 96 and 128)
    from mgkmc_b200 import checkpoint as C
    from mgkmc_b200.kmc3d import Kmc3D, in_plane_modes
    M = 8
    rng0 = np.random.default_rng(4)
    E, nu = W.ls3d_material(n, n, n, rng0)
    cat = in_plane_modes(rng0.uniform(0.0, np.pi, (n, n, n, M)), 0.1)
    Q0 = np.clip(rng0.normal(0.5, 0.15, (n, n, n, M)), 0.3, None)
    kw = dict(step_size=1e-4, q_mean=0.5, selection=selection, ls_start=ls_start, precision=precision)
    full = Kmc3D(E, nu, cat, Q0, **kw).run(np.random.default_rng(9), 40)
    a = Kmc3D(E, nu, cat, Q0, **kw)
    rng = np.random.default_rng(9)
    a.run(rng, 20)
    path = C.save_trajectory(str(tmp_path / "traj3"), a, rng)
    st, rng2, meta = C.load_trajectory(path)
    assert meta["step"] == 20 and meta["nz"] == n
    b = Kmc3D(st["E"], st["nu"], st["catalog"], st["Q0"], **kw)
    b.load_state_dict(st)
    res = b.run(rng2, 40)
    assert len(full["events"]) > 0
    assert res["events"] == full["events"]
    np.testing.assert_array_equal(res["sig"], full["sig"])
    np.testing.assert_array_equal(res["eps_p"], full["eps_p"])
    np.testing.assert_array_equal(res["eps_macro"], full["eps_macro"])
    assert res["time"] == full["time"] and res["solves"] == full["solves"]


def test_kmc3d_driver_matches_reference_trajectory(golden):
    # the reference's own 3D trajectory (ThermalSimulation.run_simulation,
    # small strain): 1348 events, identical modes, times to 1e-9
    from mgkmc_b200.kmc3d import Kmc3D, ReferenceDraws3D
    g = golden("kmc3d_traj_6x6x4")
    rs = np.random.RandomState()
    rs.set_state(("MT19937", g["rs_keys"], int(g["rs_pos"]), int(g["rs_has_gauss"]), float(g["rs_gauss"])))
    k = Kmc3D(g["E"], g["nu"], g["catalog0"], g["Q00"], T=300.0, step_size=float(g["step_size"]), jp=0.0, jt=0.0,
              cap=2.0, mixed_tol=1e4, mixed_max_iter=50)
    r = k.run(ReferenceDraws3D(rs, 0.1, 0.4, 0.15, 0.2), int(g["n_steps"]))
    np.testing.assert_array_equal(np.array([e[:4] for e in r["events"]]), g["events"])
    t = np.array([e[4] for e in r["events"]])
    assert np.max(np.abs(t - g["times"]) / np.abs(g["times"])) < 1e-9
    np.testing.assert_allclose(r["eps_macro"], g["eps_macro"], rtol=1e-9, atol=1e-15)
    assert rel(r["sig"], g["sig"]) < 1e-9
    np.testing.assert_array_equal(r["eps_p"], g["eps_plastic"])
    np.testing.assert_array_equal(r["catalog"], g["catalog"])


def test_kmc3d_driver_matches_oracle_at_32():
    # 32^3 x 8 modes, the benchmark's barrier model centred at 0.5 eV, the
    # device driver against the oracle driver with the same Generator draws
    from mgkmc_b200.kmc3d import Kmc3D
    from oracle import kmc_driver as OD
    n, M = 32, 8
    rng0 = np.random.default_rng(3)
    E, nu = W.ls3d_material(n, n, n, rng0)
    theta = rng0.uniform(0.0, np.pi, (n, n, n, M))
    cat = OD.in_plane_modes(theta, 0.1)
    Q0 = np.clip(rng0.normal(0.5, 0.15, (n, n, n, M)), 0.3, None)
    kw = dict(step_size=1e-4, q_mean=0.5)
    o = OD.run_kmc3d(E, nu, cat, Q0, np.random.default_rng(8), n_steps=30, max_events=20, **kw)
    r = Kmc3D(E, nu, cat, Q0, **kw).run(np.random.default_rng(8), 30, max_events=20)
    assert len(r["events"]) == len(o["events"]) and len(o["events"]) > 0
    for a, b in zip(r["events"], o["events"]):
        assert a[:4] == b[:4]
        assert abs(a[4] - b[4]) <= 1e-9 * abs(b[4])
    np.testing.assert_allclose(r["eps_macro"], o["eps_macro"], rtol=1e-9, atol=1e-15)
    assert rel(r["sig"], o["sig"]) < 1e-9
