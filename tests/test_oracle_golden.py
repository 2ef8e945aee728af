"""The CPU oracle restatements reproduce the unmodified reference's outputs
(golden fixtures made by tests/golden/make_golden.py)."""
import numpy as np
import pytest

from oracle import kmc as OK
from oracle import ls as OL


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("k", [1, 5])
def test_ls2d_fixed_iterations(golden, k):
    g = golden("ls2d_cfg0_64")
    eps, sig, _, _ = OL.spectral_solver(g["E"], g["nu"], g["eps_bar"], g["eps_plastic"], max_iter=k, tol=0.0)
    assert rel(eps, g[f"eps_it{k}"]) < 1e-12
    assert rel(sig, g[f"sig_it{k}"]) < 1e-12


def test_ls2d_converged(golden):
    g = golden("ls2d_cfg0_64")
    eps, sig, em, sm = OL.spectral_solver(g["E"], g["nu"], g["eps_bar"], g["eps_plastic"], max_iter=500, tol=1e-10)
    assert rel(eps, g["eps_conv"]) < 1e-12
    assert rel(sig, g["sig_conv"]) < 1e-12
    assert rel(sm, g["sig_mean"]) < 1e-12


def test_ls2d_plane_stress_warm_start_asymmetric(golden):
    g = golden("ls2d_24x16_pstress")
    for k in (1, 3):
        eps, sig, _, _ = OL.spectral_solver(g["E"], g["nu"], g["eps_bar"], g["eps_plastic"], max_iter=k,
                                            tol=0.0, plane_mode="plane_stress", eps_init=g["eps_init"])
        assert rel(eps, g[f"eps_it{k}"]) < 1e-12
        assert rel(sig, g[f"sig_it{k}"]) < 1e-12
    eps, sig, _, _ = OL.spectral_solver(g["E"], g["nu"], g["eps_bar"], g["eps_plastic"], max_iter=300,
                                        tol=1e-11, plane_mode="plane_stress", eps_init=g["eps_init"])
    assert rel(eps, g["eps_conv"]) < 1e-12


@pytest.mark.parametrize("tag", ["a", "b"])
def test_ls2d_secant(golden, tag):
    # the secant-degradation LS restatement against the reference's solver
    g = golden("ls2d_secant_24x16")
    eps, sig, _, _ = OL.spectral_solver_secant_2d(g["lam"], g["mu"], float(g[f"d_{tag}"]), float(g[f"k_{tag}"]),
                                                  g["eps_bar"], g["eps_plastic"], max_iter=500, tol=1e-12)
    assert rel(eps, g[f"eps_{tag}"]) < 1e-12
    assert rel(sig, g[f"sig_{tag}"]) < 1e-12


def test_ls2d_secant_warm(golden):
    g = golden("ls2d_secant_24x16")
    eps, sig, _, _ = OL.spectral_solver_secant_2d(g["lam"], g["mu"], 0.3, 50.0, g["eps_bar"] * 1.1, g["eps_plastic"],
                                                  max_iter=500, tol=1e-12, eps_init=g["eps_init"])
    assert rel(eps, g["eps_warm"]) < 1e-12
    assert rel(sig, g["sig_warm"]) < 1e-12


@pytest.mark.parametrize("tag", ["a", "b", "warm"])
def test_ls3d_secant(golden, tag):
    # the 3D secant-degradation LS restatement against the reference's solver
    g = golden("ls3d_secant_12x8x6")
    if tag == "warm":
        eps, sig, _, _ = OL.spectral_solver_secant_3d(g["lam"], g["mu"], 0.3, 50.0, g["eps_bar"] * 1.1,
                                                      g["eps_plastic"], max_iter=500, tol=1e-12,
                                                      eps_init=g["eps_init"])
    else:
        eps, sig, _, _ = OL.spectral_solver_secant_3d(g["lam"], g["mu"], float(g[f"d_{tag}"]),
                                                      float(g[f"k_{tag}"]), g["eps_bar"], g["eps_plastic"],
                                                      max_iter=500, tol=1e-12)
    assert rel(eps, g[f"eps_{tag}"]) < 1e-12
    assert rel(sig, g[f"sig_{tag}"]) < 1e-12


@pytest.mark.parametrize("tag,cap,limit,power", [("plain", None, None, 1.0), ("piecewise", "piecewise", 0.015, 1.0),
                                                   ("piecewise_auto", "piecewise", None, 1.0),
                                                   ("smooth", "smooth", 0.015, 2.0)])
def test_landau_law(golden, tag, cap, limit, power):
    # the Landau stress restatement against the reference's stress_from_strain_landau_2d
    g = golden("ls2d_landau_16x12")
    sig = OL.landau_stress_2d(g["strain"], g["lam"], g["mu"], tuple(g["v"]), cap, limit, 0.1, power)
    np.testing.assert_array_equal(sig, g[f"sig_{tag}"])


@pytest.mark.parametrize("tag", ["aa5", "aa0", "cap"])
def test_landau_solver(golden, tag):
    # the Landau LS restatement (basic scheme, Anderson mixing) against the reference's solver
    g = golden("ls2d_landau_16x12")
    kw = dict(anderson_m=0) if tag == "aa0" else dict(cap_type="piecewise", cap_limit=0.01) if tag == "cap" else {}
    eps, sig, _, _ = OL.spectral_solver_landau_2d(g["lam"], g["mu"], tuple(g["v"]), g["eps_bar"], g["eps_plastic"],
                                                  max_iter=400, tol=1e-12, **kw)
    assert rel(eps, g[f"eps_{tag}"]) < 1e-12
    assert rel(sig, g[f"sig_{tag}"]) < 1e-12


@pytest.mark.parametrize("tag,pm", [("ps", "plane_strain"), ("pst", "plane_stress")])
def test_ls2d_rose(golden, tag, pm):
    # the Rose-law LS restatement against the reference's solver
    g = golden("ls2d_rose_16x24")
    eps, sig, _, _ = OL.spectral_solver_rose_2d(g["lam"], g["mu"], float(g[f"eta_{tag}"]), float(g[f"floor_{tag}"]),
                                                g["eps_bar"], g["eps_plastic"], max_iter=500, tol=1e-12,
                                                plane_mode=pm)
    assert rel(eps, g[f"eps_{tag}"]) < 1e-12
    assert rel(sig, g[f"sig_{tag}"]) < 1e-12


@pytest.mark.parametrize("tag", ["t0", "t1"])
def test_find_unstable(golden, tag):
    # the cascade's unstable-mode list against the reference's find_unstable_2d
    g = golden("kmc2d_cascade_12x10")
    np.testing.assert_array_equal(OK.find_unstable_2d(g["Q"], float(g[f"thr_{tag}"])), g[f"unstable_{tag}"])


@pytest.mark.parametrize("R", [3, 9])
def test_patch_kernels(golden, R):
    # fast-patching stress patches against the reference's _precompute_patch_kernels
    # (R = 9: the 19 x 19 window wraps the 16 x 12 grid)
    from oracle import kmc_driver as OD
    g = golden("kmc2d_patch_16x12")
    kern, miss = OD.patch_kernels_2d(g["E"], g["nu"], R)
    assert rel(kern, g[f"kernels_r{R}"]) < 1e-12
    np.testing.assert_allclose(miss, g[f"missing_r{R}"], rtol=0, atol=1e-12 * np.max(np.abs(kern)))


def test_apply_patch_wrap_order():
    # the vectorised window add equals the reference's (dx, dy) loop, also when
    # the window is wider than the grid and voxels receive several adds
    from oracle import kmc_driver as OD
    rng = np.random.default_rng(5)
    nx, ny, R = 5, 4, 3
    kern = rng.normal(size=(2, 2 * R + 1, 2 * R + 1, 2, 2))
    miss = rng.normal(size=(2, 2, 2))
    sig0 = rng.normal(size=(nx, ny, 2, 2))
    unit = rng.normal(size=(nx, ny, 2, 2))
    gxx, gxy, x, y, scale = 0.031, -0.017, 4, 1, 0.37
    sig = sig0.copy()
    OD.apply_patch_2d(sig, x, y, gxx, gxy, kern, miss, unit=unit, scale=scale)
    ref = sig0 + unit * scale
    patch = gxx * kern[0] + gxy * kern[1]
    for dx in range(-R, R + 1):
        for dy in range(-R, R + 1):
            ref[(x + dx) % nx, (y + dy) % ny] += patch[dx + R, dy + R]
    ref += gxx * miss[0] + gxy * miss[1]
    np.testing.assert_array_equal(sig, ref)


def test_ls2d_macro_loop(golden):
    g = golden("ls2d_macro_16")
    E, nu, mask, target = g["E"], g["nu"], g["mask"], g["target"]
    # the reference driver ramps targets over n_steps=2 with warm starts
    eps_warm, eps_bar = None, np.zeros((2, 2))
    for s in range(3):
        t = target * (s / 2)
        eps, sig, eps_bar, sigM, _, _ = OL.mixed_bc_solve_2d(
            E, nu, None, mask, t, tol_ls=1e-10, max_iter_ls=300, tol_macro=1e3, max_iter_macro=30,
            eps_bar0=eps_bar, eps_warm=eps_warm)
        eps_warm = eps
        scale = np.max(np.abs(g["sigM"]))
        assert np.max(np.abs(sigM - g["sigM"][s])) < 1e-9 * scale
    assert rel(eps, g["eps_last"]) < 1e-9


@pytest.mark.parametrize("name", ["ls3d_8x8x8", "ls3d_12x8x6"])
def test_ls3d(golden, name):
    g = golden(name)
    eps, sig, _, _ = OL.spectral_solver(g["E"], g["nu"], g["eps_bar"], g["eps_plastic"], max_iter=2, tol=0.0)
    assert rel(eps, g["eps_it2"]) < 1e-12
    assert rel(sig, g["sig_it2"]) < 1e-12
    eps, sig, _, _ = OL.spectral_solver(g["E"], g["nu"], g["eps_bar"], g["eps_plastic"], max_iter=300, tol=1e-10)
    assert rel(eps, g["eps_conv"]) < 1e-12
    assert rel(sig, g["sig_conv"]) < 1e-12


def test_kmc2d_barrier(golden):
    g = golden("kmc2d_16x12")
    for c, (t, cap, scheme, tau, vol) in enumerate(g["cases"]):
        Q = np.zeros_like(g["Q0"])
        OK.compute_barrier(Q, g["Q0"], g["sig"], g["catalog"], vol, g["soft_prop"], g["last_event_time"],
                           t, g["prev_dir"], cap, int(scheme), tau)
        np.testing.assert_allclose(Q, g[f"Q_case{c}"], rtol=0, atol=1e-14)


def test_barrier_known_answer():
    # tests/test_barrier_physics.py:13-47 of the reference: 1 GPa shear, gamma 0.1
    sig = np.zeros((1, 1, 1, 3, 3)); sig[0, 0, 0, 0, 1] = sig[0, 0, 0, 1, 0] = 1e9
    cat = np.zeros((1, 1, 1, 1, 3, 3)); cat[0, 0, 0, 0, 0, 1] = cat[0, 0, 0, 0, 1, 0] = 0.1
    Q = np.zeros((1, 1, 1, 1))
    OK.compute_barrier(Q, np.ones((1, 1, 1, 1)), sig, cat, 1.0, np.zeros((1, 1, 1, 4)),
                       np.full((1, 1, 1), -np.inf), 0.0, np.zeros((1, 1, 1, 3, 3)), 2.0, 0, np.inf)
    assert abs(Q[0, 0, 0, 0] - (1.0 - 0.6241509)) < 1e-4


def test_kmc2d_rates_exact(golden):
    g = golden("kmc2d_16x12")
    Q = g["Q_rates"]
    for T in (300.0, 0.0):
        for cm in (False, True):
            tag = f"T{int(T)}_c{int(cm)}"
            r, idx, total = OK.compute_rates(Q, 1.0, T, 1e13, cascade_mode=cm)
            np.testing.assert_array_equal(idx, g[f"indices_{tag}"])
            np.testing.assert_allclose(r, g[f"rates_{tag}"], rtol=1e-15, atol=0)  # exp() differs by <= 1 ulp across libms
            # total is the sequential sum of the reference's own rates: bit-exact
            assert np.add.accumulate(g[f"rates_{tag}"])[-1] == g[f"total_{tag}"]


def test_kmc2d_select_bit_exact(golden):
    g = golden("kmc2d_16x12")
    rates, total = g["rates_T300_c0"], float(g["total_T300_c0"])
    for u, k in zip(g["sel_u"], g["sel_idx"]):
        assert OK.select_event(rates, total, u) == k
        assert OK.select_event_loop(rates, total, u) == k


def test_kmc2d_flip_bit_exact(golden):
    g = golden("kmc2d_16x12")
    ep, sp, tl = g["flip_in_eps_p"].copy(), g["flip_in_soft"].copy(), g["flip_in_tlast"].copy()
    for (x, y, m, t, jp, jt, gmax, jn) in g["flips"]:
        OK.apply_flip_2d(ep, sp, tl, g["catalog"], int(x), int(y), int(m), t, jp, jt, gmax, jn)
    np.testing.assert_array_equal(ep, g["flip_out_eps_p"])
    np.testing.assert_array_equal(sp, g["flip_out_soft"])
    np.testing.assert_array_equal(tl, g["flip_out_tlast"])


def test_kmc3d(golden):
    g = golden("kmc3d_6x5x4")
    Q = np.zeros_like(g["Q0"])
    OK.compute_barrier(Q, g["Q0"], g["sig"], g["catalog"], 1.0, g["soft_prop"], g["last_event_time"],
                       1e-3, g["prev_dir"], 0.5, 1, 5e-4)
    np.testing.assert_allclose(Q, g["Q"], rtol=0, atol=1e-14)
    Q2 = np.zeros_like(g["Q0"])
    OK.compute_barrier(Q2, g["Q0"], g["sig"], g["catalog"], 1.0, g["soft_prop"], g["last_event_time"],
                       1e-3, g["prev_dir"], 0.5, 0, np.inf)
    np.testing.assert_allclose(Q2, g["Q_iso"], rtol=0, atol=1e-14)
    r, idx, total = OK.compute_rates(g["Q"], 1.0, 300.0, 1e13, cascade_mode=False)
    np.testing.assert_array_equal(idx, g["indices"])
    for u, k in zip(g["sel_u"], g["sel_idx"]):
        assert OK.select_event(g["rates"], float(g["total"]), u) == k
    ep, sp, tl = g["flip_in_eps_p"].copy(), g["flip_in_soft"].copy(), g["flip_in_tlast"].copy()
    for (x, y, z, m, t, jp, jt, gmax, jn) in g["flips"]:
        OK.apply_flip_3d(ep, sp, tl, g["catalog"], int(x), int(y), int(z), int(m), t, jp, jt, gmax, jn)
    np.testing.assert_array_equal(ep, g["flip_out_eps_p"])
    np.testing.assert_array_equal(sp, g["flip_out_soft"])
    np.testing.assert_array_equal(tl, g["flip_out_tlast"])


def _reference_draws(g, mod):
    rs = np.random.RandomState()
    rs.set_state(("MT19937", g["rs_keys"], int(g["rs_pos"]), int(g["rs_has_gauss"]), float(g["rs_gauss"])))
    return mod.ReferenceDraws(rs, 0.1, 0.6, 0.15, 0.3)


def test_kmc_driver_matches_reference_trajectory(golden):
    # the reference's own KmcSimulation2D.run_simulation trajectory (174 events
    # over 60 AQS steps), reproduced from the same initial catalog, barriers
    # and RandomState draws
    from oracle import kmc_driver as OD
    g = golden("kmc2d_traj_12x8")
    o = OD.run_kmc2d(g["E"], g["nu"], g["catalog0"], g["Q00"], _reference_draws(g, OD), n_steps=int(g["n_steps"]),
                     step_size=float(g["step_size"]), strain_rate=1e7, T=300.0, jp=0.0, jt=0.0, cap=2.0,
                     mixed_tol=1e4, mixed_max_iter=50, ls_tol=1e-6, ls_max_iter=200)
    assert len(o["events"]) == len(g["events"])
    np.testing.assert_array_equal(np.array([e[:3] for e in o["events"]]), g["events"])
    t = np.array([e[3] for e in o["events"]])
    assert np.max(np.abs(t - g["times"]) / np.abs(g["times"])) < 1e-12
    assert np.max(np.abs(o["eps_macro"] - g["eps_macro"])) < 1e-15
    assert rel(o["sig"], g["sig"]) < 1e-12
    np.testing.assert_array_equal(o["eps_p"], g["eps_plastic"])
    np.testing.assert_array_equal(o["catalog"], g["catalog"])
    np.testing.assert_array_equal(o["Q0"], g["Q0"])


def test_kmc3d_driver_matches_reference_trajectory(golden):
    # the reference's own ThermalSimulation.run_simulation trajectory (small
    # strain, 1348 events over 60 AQS steps on 6x6x4 x 4 modes)
    from oracle import kmc_driver as OD
    g = golden("kmc3d_traj_6x6x4")
    rs = np.random.RandomState()
    rs.set_state(("MT19937", g["rs_keys"], int(g["rs_pos"]), int(g["rs_has_gauss"]), float(g["rs_gauss"])))
    o = OD.run_kmc3d(g["E"], g["nu"], g["catalog0"], g["Q00"], OD.ReferenceDraws3D(rs, 0.1, 0.4, 0.15, 0.2),
                     n_steps=int(g["n_steps"]), step_size=float(g["step_size"]), T=300.0, jp=0.0, jt=0.0, cap=2.0,
                     mixed_tol=1e4, mixed_max_iter=50)
    np.testing.assert_array_equal(np.array([e[:4] for e in o["events"]]), g["events"])
    t = np.array([e[4] for e in o["events"]])
    assert np.max(np.abs(t - g["times"]) / np.abs(g["times"])) < 1e-12
    assert np.max(np.abs(o["eps_macro"] - g["eps_macro"])) < 1e-15
    assert rel(o["sig"], g["sig"]) < 1e-12
    np.testing.assert_array_equal(o["eps_p"], g["eps_plastic"])
    np.testing.assert_array_equal(o["catalog"], g["catalog"])
    np.testing.assert_array_equal(o["Q0"], g["Q0"])


def test_landau_3d_law_and_solver(golden):
    # the reference's 3D Landau law (plain, piecewise and smooth capping) and
    # its basic-scheme LS solver at fixed iteration counts and converged
    g = golden("ls3d_landau_12x8x6")
    v = tuple(g["v"])
    e = g["strain"]
    assert rel(OL.landau_stress_3d(e, g["lam"], g["mu"], v), g["sig_plain"]) < 1e-13
    assert rel(OL.landau_stress_3d(e, g["lam"], g["mu"], v, "piecewise", 0.015), g["sig_piecewise"]) < 1e-13
    assert rel(OL.landau_stress_3d(e, g["lam"], g["mu"], v, "smooth", 0.015, cap_power=2.0), g["sig_smooth"]) < 1e-13
    kw = dict(eps_plastic=g["eps_plastic"])
    for k in (1, 3):
        eps, sig, _, _ = OL.spectral_solver_landau_3d(g["lam"], g["mu"], v, g["eps_bar"], max_iter=k, tol=0.0, **kw)
        assert rel(eps, g[f"eps_it{k}"]) < 1e-12 and rel(sig, g[f"sig_it{k}"]) < 1e-12
    eps, sig, _, _ = OL.spectral_solver_landau_3d(g["lam"], g["mu"], v, g["eps_bar"], max_iter=400, tol=1e-12, **kw)
    assert rel(eps, g["eps_conv"]) < 1e-12 and rel(sig, g["sig_conv"]) < 1e-12
    eps, sig, _, _ = OL.spectral_solver_landau_3d(g["lam"], g["mu"], v, g["eps_bar"], max_iter=400, tol=1e-12,
                                                  cap_type="smooth", cap_limit=0.01, cap_power=2.0, **kw)
    assert rel(eps, g["eps_cap"]) < 1e-12 and rel(sig, g["sig_cap"]) < 1e-12


def test_landau_plane_stress_law_and_solver(golden):
    # the oracle's plane-stress Landau law (global e33 Newton, warm state) and
    # solver against the reference's
    from oracle import ls as OL
    g = golden("ls2d_landau_pstress_16x12")
    v = tuple(g["v"])
    caps = {"plain": (None, None, 1.0), "piecewise": ("piecewise", 0.015, 1.0), "smooth": ("smooth", 0.015, 2.0)}
    for tag, (ct, cl, cp) in caps.items():
        st = {}
        sig = OL.landau_stress_2d(g["strain"], g["lam"], g["mu"], v, ct, cl, 0.1, cp, True, st)
        assert np.max(np.abs(sig - g[f"sig_{tag}"])) <= 1e-12 * np.max(np.abs(g[f"sig_{tag}"]))
        assert np.max(np.abs(st["e33"] - g[f"e33_{tag}"])) <= 1e-15
        warm = {"e33": g[f"warm_in_{tag}"].copy()}
        sig = OL.landau_stress_2d(g["strain"], g["lam"], g["mu"], v, ct, cl, 0.1, cp, True, warm)
        assert np.max(np.abs(sig - g[f"sig_warm_{tag}"])) <= 1e-12 * np.max(np.abs(g[f"sig_warm_{tag}"]))
    for tag, (ct, cl) in (("solve", (None, None)), ("solve_cap", ("piecewise", 0.01))):
        st = {}
        o = OL.spectral_solver_landau_2d(g["lam"], g["mu"], v, g["eps_bar"], g["eps_plastic"], max_iter=400, tol=1e-12,
                                         anderson_m=5, cap_type=ct, cap_limit=cl, plane_stress=True, e33_state=st)
        assert np.max(np.abs(o[0] - g[f"eps_{tag}"])) < 1e-9 * np.max(np.abs(g[f"eps_{tag}"]))
        assert np.max(np.abs(o[1] - g[f"sig_{tag}"])) < 1e-9 * np.max(np.abs(g[f"sig_{tag}"]))


def test_landau_plane_stress_root_fixed_point_matches_reference(golden):
    # e33 solved to its root at every evaluation (as the GPU kernels do)
    # reaches the reference's fixed point within 1e-9 on its own fixtures
    from oracle import ls as OL
    g = golden("ls2d_landau_pstress_16x12")
    v = tuple(g["v"])
    for tag, (ct, cl) in (("solve", (None, None)), ("solve_cap", ("piecewise", 0.01))):
        o = OL.spectral_solver_landau_2d(g["lam"], g["mu"], v, g["eps_bar"], g["eps_plastic"], max_iter=400, tol=1e-12,
                                         anderson_m=5, cap_type=ct, cap_limit=cl, plane_stress=True, e33_root=True)
        assert np.max(np.abs(o[0] - g[f"eps_{tag}"])) < 1e-9 * np.max(np.abs(g[f"eps_{tag}"]))
        assert np.max(np.abs(o[1] - g[f"sig_{tag}"])) < 1e-9 * np.max(np.abs(g[f"sig_{tag}"]))
