"""Generate golden fixtures by running the UNMODIFIED reference mgkmc code.

Run in a container that has the reference checkout (default /root/reference,
override with MGKMC_REFERENCE):

    python tests/golden/make_golden.py

Each fixture is an .npz of seeded inputs and the reference's outputs for one
hot-path function.  The reference imports pyfftw/h5py/meshio/matplotlib at
module level; ``oracle.ref_import`` maps pyfftw onto numpy.fft and stubs the
I/O modules (none of which the hot path uses).  Numba kernels whose selection
draws come from numba's private RNG are run through ``.py_func`` under
``np.random.seed`` so the uniform draw is reproducible and recorded.

Fixtures are small (grids up to 64^2 / 8^3) so the repository stays light; the
GPU parity tests rerun the oracle at larger sizes.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.abspath(os.path.join(HERE, "..", "..")))

from oracle.ref_import import import_reference  # noqa: E402
from mgkmc_b200 import workloads as W  # noqa: E402

import_reference(os.environ.get("MGKMC_REFERENCE", "/root/reference"))
from mgkmc import linear_elastic_simulator as LES  # noqa: E402
from mgkmc import kmc_simulator_functions as KF  # noqa: E402
from mgkmc import finite_strain_simulator as FS  # noqa: E402
from mgkmc.stz import barriers as SB, kmc as SK, cascade as SC  # noqa: E402


def save(name, **arrays):
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **arrays)
    print(f"wrote {path} ({os.path.getsize(path)/1024:.1f} KB)")


def ls2d_fixtures():
    # config[0]: 64^2 plane strain, 5 % pure-shear eigenstrains, eps_xx = 0.01
    E, nu, ep, eb = W.ls2d_problem(64, 64, 0)
    out = {"E": E, "nu": nu, "eps_plastic": ep, "eps_bar": eb}
    for k in (1, 5):
        eps, sig, em, sm = LES.spectral_solver_2d(E, nu, eb, ep, max_iter=k, tol=0.0)
        out[f"eps_it{k}"] = eps
        out[f"sig_it{k}"] = sig
    eps, sig, em, sm = LES.spectral_solver_2d(E, nu, eb, ep, max_iter=500, tol=1e-10)
    out.update(eps_conv=eps, sig_conv=sig, eps_mean=em, sig_mean=sm)
    save("ls2d_cfg0_64", **out)

    # non-square radix-3 grid, plane stress, asymmetric eps_bar and a warm start
    rng = np.random.default_rng(11)
    E, nu = W.ls2d_material(24, 16, rng)
    ep = W.pure_shear_eigenstrain_2d(24, 16, rng, frac=0.1)
    ep[3, 5, 0, 1] += 0.01  # one asymmetric eigenstrain entry
    eb = np.array([[0.004, 0.003], [-0.001, -0.002]])
    eps_init = 1e-3 * rng.standard_normal((24, 16, 2, 2))
    out = {"E": E, "nu": nu, "eps_plastic": ep, "eps_bar": eb, "eps_init": eps_init}
    for k in (1, 3):
        eps, sig, _, _ = LES.spectral_solver_2d(E, nu, eb, ep, max_iter=k, tol=0.0,
                                                plane_mode="plane_stress", eps_init=eps_init)
        out[f"eps_it{k}"] = eps
        out[f"sig_it{k}"] = sig
    eps, sig, em, sm = LES.spectral_solver_2d(E, nu, eb, ep, max_iter=300, tol=1e-11,
                                              plane_mode="plane_stress", eps_init=eps_init)
    out.update(eps_conv=eps, sig_conv=sig, eps_mean=em, sig_mean=sm)
    save("ls2d_24x16_pstress", **out)

    # macro mixed-BC driver (no eigenstrain: the reference driver has none)
    rng = np.random.default_rng(12)
    E, nu = W.ls2d_material(16, 16, rng)
    mask = np.array([[True, True], [True, False]])
    target = np.array([[0.01, 0.0], [0.0, 0.0]])
    epsM, sigM, eps_l, sig_l = LES.linear_elastic_simulation_2d(
        E, nu, mask, target, n_steps=2, tol_ls=1e-10, max_iter_ls=300, tol_macro=1e3,
        max_iter_macro=30, enable_console=False)
    save("ls2d_macro_16", E=E, nu=nu, mask=mask, target=target, epsM=np.array(epsM),
         sigM=np.array(sigM), eps_last=eps_l[-1], sig_last=sig_l[-1])


def ls3d_fixtures():
    rng = np.random.default_rng(21)
    for shape in ((8, 8, 8), (12, 8, 6)):
        E, nu = W.ls3d_material(*shape, rng)
        ep = W.pure_shear_eigenstrain_3d(*shape, rng, frac=0.05)
        eb = np.zeros((3, 3))
        eb[0, 0] = 0.01
        eb[1, 2] = eb[2, 1] = 0.002
        out = {"E": E, "nu": nu, "eps_plastic": ep, "eps_bar": eb}
        eps, sig, _, _ = LES.spectral_solver_3d(E, nu, eb, ep, max_iter=2, tol=0.0)
        out.update(eps_it2=eps, sig_it2=sig)
        eps, sig, em, sm = LES.spectral_solver_3d(E, nu, eb, ep, max_iter=300, tol=1e-10)
        out.update(eps_conv=eps, sig_conv=sig, eps_mean=em, sig_mean=sm)
        save("ls3d_%dx%dx%d" % shape, **out)


def kmc2d_fixtures():
    rng = np.random.default_rng(31)
    nx, ny, M = 16, 12, 8
    cat, Q0 = W.kmc2d_state(nx, ny, M, rng)
    cat[2, 3, 1, 0, 1] += 0.02  # one asymmetric mode
    sig = 1e9 * rng.standard_normal((nx, ny, 2, 2))
    soft = np.abs(0.2 * rng.standard_normal((nx, ny, 2)))
    soft[rng.random((nx, ny)) < 0.5, 1] = 0.0
    t_last = np.where(rng.random((nx, ny)) < 0.3, -np.inf, rng.uniform(0, 1e-3, (nx, ny)))
    prev = 0.05 * rng.standard_normal((nx, ny, 2, 2))
    prev[rng.random((nx, ny)) < 0.4] = 0.0
    out = {"catalog": cat, "Q0": Q0, "sig": sig, "soft_prop": soft, "last_event_time": t_last,
           "prev_dir": prev}
    cases = [  # (time, cap, scheme, tau, volume)
        (1e-3, 0.5, 0, np.inf, 1.0),
        (2e-3, 0.3, 1, 5e-4, 0.343),
        (0.0, 0.0, 0, 1e-3, 1.0),
    ]
    for c, (t, cap, scheme, tau, vol) in enumerate(cases):
        Q = np.zeros((nx, ny, M))
        KF.compute_barrier_2d(Q, Q0, sig, cat, vol, soft, t_last, t, prev, cap, scheme, tau)
        out[f"Q_case{c}"] = Q
    out["cases"] = np.array([[t, cap, scheme, tau, vol] for (t, cap, scheme, tau, vol) in cases])
    Q = out["Q_case1"].copy()
    Q[0, 0, :3] = -0.1  # a few unstable modes
    Q[5, 5, 2] = 0.0
    out["Q_rates"] = Q
    for T in (300.0, 0.0):
        for cm in (False, True):
            rates, idx, total = KF.compute_rates_2d(Q, 1.0, T, 1e13, cascade_mode=cm)
            tag = f"T{int(T)}_c{int(cm)}"
            out[f"rates_{tag}"] = rates
            out[f"indices_{tag}"] = idx
            out[f"total_{tag}"] = np.array(total)
    rates, idx, total = KF.compute_rates_2d(Q, 1.0, 300.0, 1e13, cascade_mode=False)
    draws, sel = [], []
    for s in range(64):
        np.random.seed(1000 + s)
        k = KF.select_event_2d.py_func(rates, total)
        np.random.seed(1000 + s)
        u = np.random.random_sample()
        draws.append(u)
        sel.append(k)
    out["sel_u"] = np.array(draws)
    out["sel_idx"] = np.array(sel)
    # explicit edge draws: exact partial-sum hits and the top of the range
    S = np.cumsum(rates)
    out["sel_total_seq"] = np.array(total)
    assert S[-1] == total
    # flips
    ep = 0.01 * rng.standard_normal((nx, ny, 2, 2))
    sp = np.abs(0.1 * rng.standard_normal((nx, ny, 2)))
    tl = rng.uniform(0, 1, (nx, ny))
    flips = [(3, 4, 2, 0.5, 10.0, 30.0, 2.0, 0.0), (0, 11, 7, 0.7, 10.0, 30.0, 0.3, 0.25),
             (15, 0, 0, 0.9, 5.0, 0.0, 0.0, 0.5)]
    out["flip_in_eps_p"], out["flip_in_soft"], out["flip_in_tlast"] = ep.copy(), sp.copy(), tl.copy()
    for (x, y, m, t, jp, jt, gmax, jn) in flips:
        KF.apply_flip_soa_2d.py_func(ep, sp, tl, cat, x, y, m, t, jp, jt, gmax, jn)
    out["flips"] = np.array(flips)
    out["flip_out_eps_p"], out["flip_out_soft"], out["flip_out_tlast"] = ep, sp, tl
    save("kmc2d_16x12", **out)


def kmc3d_fixtures():
    rng = np.random.default_rng(41)
    nx, ny, nz, M = 6, 5, 4, 6
    cat = 0.05 * rng.standard_normal((nx, ny, nz, M, 3, 3))
    Q0 = np.clip(rng.normal(1.0, 0.15, (nx, ny, nz, M)), 0.3, None)
    sig = 1e9 * rng.standard_normal((nx, ny, nz, 3, 3))
    soft = np.abs(0.2 * rng.standard_normal((nx, ny, nz, 4)))
    t_last = np.where(rng.random((nx, ny, nz)) < 0.3, -np.inf, rng.uniform(0, 1e-3, (nx, ny, nz)))
    prev = 0.05 * rng.standard_normal((nx, ny, nz, 3, 3))
    out = {"catalog": cat, "Q0": Q0, "sig": sig, "soft_prop": soft, "last_event_time": t_last,
           "prev_dir": prev}
    Q = np.zeros((nx, ny, nz, M))
    SB.compute_barrier(Q, Q0, sig, cat, 1.0, soft, t_last, 1e-3, prev, 0.5, 1, 5e-4)
    out["Q"] = Q.copy()
    Q2 = np.zeros((nx, ny, nz, M))
    SB.compute_barrier(Q2, Q0, sig, cat, 1.0, soft, t_last, 1e-3, prev, 0.5, 0, np.inf)
    out["Q_iso"] = Q2
    rates, idx, total = SK.compute_rates(Q, 1.0, 300.0, 1e13, cascade_mode=False)
    out.update(rates=rates, indices=idx, total=np.array(total))
    draws, sel = [], []
    for s in range(32):
        np.random.seed(2000 + s)
        k = SK.select_event.py_func(rates, total)
        np.random.seed(2000 + s)
        draws.append(np.random.random_sample())
        sel.append(k)
    out["sel_u"], out["sel_idx"] = np.array(draws), np.array(sel)
    ep = 0.01 * rng.standard_normal((nx, ny, nz, 3, 3))
    sp = np.abs(0.1 * rng.standard_normal((nx, ny, nz, 4)))
    tl = rng.uniform(0, 1, (nx, ny, nz))
    out["flip_in_eps_p"], out["flip_in_soft"], out["flip_in_tlast"] = ep.copy(), sp.copy(), tl.copy()
    flips = [(1, 2, 3, 4, 0.5, 10.0, 30.0, 2.0, 0.2), (5, 0, 0, 0, 0.6, 10.0, 30.0, 0.3, 0.0)]
    for (x, y, z, m, t, jp, jt, gmax, jn) in flips:
        SC.apply_flip_soa.py_func(ep, None, sp, tl, cat, x, y, z, m, t, jp, jt, gmax, jn)
    out["flips"] = np.array(flips)
    out["flip_out_eps_p"], out["flip_out_soft"], out["flip_out_tlast"] = ep, sp, tl
    save("kmc3d_6x5x4", **out)


def fs3d_fixtures():
    """One mixed-BC load step of the reference Newton-Krylov solver (SVK + F_p)."""
    rng = np.random.default_rng(51)
    nx = ny = nz = 6
    E, nu, Fp = W.fs3d_material(nx, ny, nz, rng, fp_frac=0.1)
    Ghat4 = FS.build_ghat4_3d(nx, ny, nz, nx * 1.0, ny * 1.0, nz * 1.0)
    I2, I4, I4rt, I4s, II = FS._make_identity_tensors_3d(nx, ny, nz)
    C4 = FS.build_C4_3d(E, nu, I4s, II)
    F0 = np.einsum("ij,xyz->ijxyz", np.eye(3), np.ones((nx, ny, nz)))
    out = {"E": E, "nu": nu, "Fp": Fp}
    F_bar, F_mask, P_tgt, P_mask = FS.build_finite_strain_bc_3d(
        (0, 0), 0.01, {(1, 1): 0.0, (2, 2): 0.0}, ndim=3)
    F, P, Sig, K4, Fb = FS.finite_strain_solver_step_3d(
        F0, F_bar, Ghat4, C4, I2, I4, I4rt, Fp=Fp, driving_component=(0, 0),
        P_target=P_tgt, P_mask=P_mask, E_avg=E.mean(), nu_avg=nu.mean(),
        tol_NW=1e-10, tol_CG=1e-10, max_NW=30, tol_macro=1e3, max_iter_macro=30,
        enable_console=False, model_type="svk", solver="newton_cg")
    out.update(F_bar_in=F_bar, P_mask=P_mask, F=F, P=P, Sig=Sig, F_bar_out=Fb)
    # constitutive law alone (SVK, with F_p) at a perturbed F
    Ft = F0 + 0.01 * rng.standard_normal(F0.shape)
    Pc, K4c = FS.constitutive_hyperelastic_3d(Ft, C4, I2, I4, I4rt, Fp=Fp, model_type="svk")
    dF = rng.standard_normal(F0.shape)
    KdF = np.einsum("ijxyz->jixyz", np.einsum("ijklxyz,lkxyz->ijxyz", K4c,
                                              np.einsum("ijxyz->jixyz", dF)))
    GKdF = FS._project_3d(KdF, Ghat4)
    out.update(F_trial=Ft, P_trial=Pc, dF=dF, KdF=KdF, GKdF=GKdF)
    save("fs3d_svk_6", **out)

    # 2D plane-strain Neo-Hookean law (the form restated in 3D by the oracle)
    nx2 = ny2 = 5
    E2, nu2 = W.ls2d_material(nx2, ny2, rng)
    I2b, I4b, I4rtb, I4sb, IIb = FS._make_identity_tensors_2d(nx2, ny2)
    C42 = FS.build_C4_2d(E2, nu2, I4sb, IIb)
    F2 = np.einsum("ij,xy->ijxy", np.eye(2), np.ones((nx2, ny2))) + 0.02 * rng.standard_normal((2, 2, nx2, ny2))
    P2, K42, _ = FS.constitutive_hyperelastic_2d(F2, C42, I2b, I4b, I4rtb, model_type="neo_hookean")
    save("fs2d_neohookean_5", E=E2, nu=nu2, F=F2, P=P2, K4=K42)


def ls2d_secant_fixtures():
    """The reference's secant-degradation LS solver (spectral_solver_secant_2d)
    on a heterogeneous medium with eigenstrains, warm and cold starts."""
    rng = np.random.default_rng(61)
    nx, ny = 24, 16
    E, nu = W.ls2d_material(nx, ny, rng)
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    ep = W.pure_shear_eigenstrain_2d(nx, ny, rng, frac=0.1)
    eb = np.array([[0.02, 0.0], [0.0, -0.005]])
    out = dict(lam=lam, mu=mu, eps_plastic=ep, eps_bar=eb)
    for tag, d, k in (("a", 0.3, 50.0), ("b", 0.8, 200.0)):
        e, s, em, sm = LES.spectral_solver_secant_2d(lam, mu, d, k, eb, eps_plastic=ep, max_iter=500, tol=1e-12)
        out.update({f"eps_{tag}": e, f"sig_{tag}": s, f"d_{tag}": d, f"k_{tag}": k})
    init = out["eps_a"] + 1e-4 * rng.standard_normal(out["eps_a"].shape)
    e, s, _, _ = LES.spectral_solver_secant_2d(lam, mu, 0.3, 50.0, eb * 1.1, eps_plastic=ep, max_iter=500, tol=1e-12,
                                               eps_init=init)
    out.update(eps_init=init, eps_warm=e, sig_warm=s)
    save("ls2d_secant_24x16", **out)


def ls3d_secant_fixtures():
    """The reference's 3D secant-degradation LS solver (spectral_solver_secant_3d)
    on a heterogeneous medium with eigenstrains, cold and warm starts."""
    rng = np.random.default_rng(67)
    shape = (12, 8, 6)
    E, nu = W.ls3d_material(*shape, rng)
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    ep = W.pure_shear_eigenstrain_3d(*shape, rng, frac=0.1)
    eb = np.zeros((3, 3))
    eb[0, 0], eb[1, 1] = 0.015, -0.004
    eb[0, 2] = eb[2, 0] = 0.003
    out = dict(lam=lam, mu=mu, eps_plastic=ep, eps_bar=eb)
    for tag, d, k in (("a", 0.3, 50.0), ("b", 0.8, 200.0)):
        e, s, _, _ = LES.spectral_solver_secant_3d(lam, mu, d, k, eb, eps_plastic=ep, max_iter=500, tol=1e-12)
        out.update({f"eps_{tag}": e, f"sig_{tag}": s, f"d_{tag}": d, f"k_{tag}": k})
    init = out["eps_a"] + 1e-4 * rng.standard_normal(out["eps_a"].shape)
    e, s, _, _ = LES.spectral_solver_secant_3d(lam, mu, 0.3, 50.0, eb * 1.1, eps_plastic=ep, max_iter=500,
                                               tol=1e-12, eps_init=init)
    out.update(eps_init=init, eps_warm=e, sig_warm=s)
    save("ls3d_secant_12x8x6", **out)


LANDAU_V = (-199.7e9, -75.4e9, -23.1e9, 1432.0e9, 311.0e9, 145.0e9, -273.0e9)  # v1 v2 v3 g1 g2 g3 g4


def ls2d_landau_fixtures():
    """The reference's Landau stress law (stress_from_strain_landau_2d, plane
    strain) without capping, with piecewise and with smooth capping, and its
    LS solver (spectral_solver_landau_2d, basic scheme with Anderson mixing of
    depth 5 and without) on a heterogeneous medium with eigenstrains."""
    from mgkmc import elasticity as ELA
    rng = np.random.default_rng(73)
    nx, ny = 16, 12
    E, nu = W.ls2d_material(nx, ny, rng)
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    v1, v2, v3, g1, g2, g3, g4 = LANDAU_V
    kw = dict(v1=v1, v2=v2, v3=v3, g1=g1, g2=g2, g3=g3, g4=g4)
    e = rng.normal(0, 0.02, (nx, ny, 2, 2))
    out = dict(lam=lam, mu=mu, v=np.array(LANDAU_V), strain=e)
    out["sig_plain"] = ELA.stress_from_strain_landau_2d(e, lam, mu, **kw)
    out["sig_piecewise"] = ELA.stress_from_strain_landau_2d(e, lam, mu, **kw, strain_capping_enabled=True,
                                                            strain_capping_limit=0.015)
    out["sig_piecewise_auto"] = ELA.stress_from_strain_landau_2d(e, lam, mu, **kw, strain_capping_enabled=True)
    out["sig_smooth"] = ELA.stress_from_strain_landau_2d(e, lam, mu, **kw, strain_capping_enabled=True,
                                                         strain_capping_limit=0.015, strain_capping_type="smooth",
                                                         strain_capping_smooth_power=2.0)
    ep = W.pure_shear_eigenstrain_2d(nx, ny, rng, frac=0.1)
    eb = np.array([[0.008, 0.002], [0.002, -0.003]])
    out.update(eps_plastic=ep, eps_bar=eb)
    for tag, m in (("aa5", 5), ("aa0", 0)):
        eps, sig, _, _ = LES.spectral_solver_landau_2d(lam, mu, **kw, eps_bar=eb, eps_plastic=ep, max_iter=400,
                                                       tol=1e-12, anderson_m=m)
        out.update({f"eps_{tag}": eps, f"sig_{tag}": sig})
    eps, sig, _, _ = LES.spectral_solver_landau_2d(lam, mu, **kw, eps_bar=eb, eps_plastic=ep, max_iter=400,
                                                   tol=1e-12, strain_capping_enabled=True,
                                                   strain_capping_limit=0.01)
    out.update(eps_cap=eps, sig_cap=sig)
    save("ls2d_landau_16x12", **out)


def ls2d_landau_pstress_fixtures():
    """The reference's Landau law in plane stress (stress_from_strain_landau_2d
    with its e33 Newton solve, elasticity.py:571-616) without capping, with
    piecewise and with smooth capping, cold and from a warm e33 state; its LS
    solver in plane stress (spectral_solver_landau_2d, basic scheme, Anderson
    depth 5, an e33 state carried across the iterations) without and with
    capping."""
    from mgkmc import elasticity as ELA
    rng = np.random.default_rng(74)
    nx, ny = 16, 12
    E, nu = W.ls2d_material(nx, ny, rng)
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    v1, v2, v3, g1, g2, g3, g4 = LANDAU_V
    kw = dict(v1=v1, v2=v2, v3=v3, g1=g1, g2=g2, g3=g3, g4=g4, plane_mode="plane_stress")
    e = rng.normal(0, 0.02, (nx, ny, 2, 2))
    e[..., 1, 0] = e[..., 0, 1]
    out = dict(lam=lam, mu=mu, v=np.array(LANDAU_V), strain=e)
    caps = {"plain": {}, "piecewise": dict(strain_capping_enabled=True, strain_capping_limit=0.015),
            "smooth": dict(strain_capping_enabled=True, strain_capping_limit=0.015, strain_capping_type="smooth",
                           strain_capping_smooth_power=2.0)}
    for tag, ck in caps.items():
        st = {}
        out[f"sig_{tag}"] = ELA.stress_from_strain_landau_2d(e, lam, mu, **kw, **ck, e33_state=st)
        out[f"e33_{tag}"] = st["e33"]
        warm = {"e33": st["e33"] + 1e-4 * rng.standard_normal(st["e33"].shape)}
        out[f"warm_in_{tag}"] = warm["e33"].copy()
        out[f"sig_warm_{tag}"] = ELA.stress_from_strain_landau_2d(e, lam, mu, **kw, **ck, e33_state=warm)
    ep = W.pure_shear_eigenstrain_2d(nx, ny, rng, frac=0.1)
    eb = np.array([[0.008, 0.002], [0.002, -0.003]])
    out.update(eps_plastic=ep, eps_bar=eb)
    for tag, ck in (("solve", {}), ("solve_cap", dict(strain_capping_enabled=True, strain_capping_limit=0.01))):
        st = {}
        eps, sig, _, _ = LES.spectral_solver_landau_2d(lam, mu, **kw, **ck, eps_bar=eb, eps_plastic=ep, max_iter=400,
                                                       tol=1e-12, anderson_m=5, e33_state=st)
        out.update({f"eps_{tag}": eps, f"sig_{tag}": sig, f"e33_{tag}": st["e33"]})
    save("ls2d_landau_pstress_16x12", **out)


def vtk_fixtures():
    """The reference's node-displacement reconstruction of its VTK writer
    (analysis/vtk.py:4-116) for a 2D and a 3D random strain field."""
    from mgkmc.analysis import vtk as RV
    rng = np.random.default_rng(75)
    e2 = rng.normal(0, 0.01, (6, 5, 2, 2))
    e3 = rng.normal(0, 0.01, (4, 3, 5, 3, 3))
    save("vtk_displacement", eps2=e2, u2=RV.reconstruct_displacement_element_centered(e2, pixel=1.5),
         eps3=e3, u3=RV.reconstruct_displacement_element_centered(e3, pixel=0.5))


def ls2d_rose_fixtures():
    """The reference's Rose-law LS solver (spectral_solver_rose_2d), plane
    strain and plane stress, with the 3D Lame lambda as its KMC driver passes."""
    rng = np.random.default_rng(62)
    nx, ny = 16, 24
    E, nu = W.ls2d_material(nx, ny, rng)
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    ep = W.pure_shear_eigenstrain_2d(nx, ny, rng, frac=0.1)
    eb = np.array([[0.02, 0.003], [0.003, -0.004]])
    out = dict(lam=lam, mu=mu, eps_plastic=ep, eps_bar=eb)
    for tag, eta, fl, pm in (("ps", 30.0, 0.1, "plane_strain"), ("pst", 60.0, 0.2, "plane_stress")):
        e, s, em, sm = LES.spectral_solver_rose_2d(lam, mu, eta, fl, eps_bar=eb, eps_plastic=ep, max_iter=500,
                                                   tol=1e-12, plane_mode=pm)
        out.update({f"eps_{tag}": e, f"sig_{tag}": s, f"eta_{tag}": eta, f"floor_{tag}": fl})
    save("ls2d_rose_16x24", **out)


def kmc2d_cascade_fixtures():
    """The reference's find_unstable_2d on a barrier field with unstable modes."""
    rng = np.random.default_rng(63)
    Q = rng.normal(0.3, 0.25, (12, 10, 4))
    out = dict(Q=Q)
    for tag, thr in (("t0", 0.0), ("t1", 0.1)):
        out[f"unstable_{tag}"] = KF.find_unstable_2d(Q, thr)
        out[f"thr_{tag}"] = thr
    save("kmc2d_cascade_12x10", **out)


def kmc2d_patch_fixtures():
    """The reference's fast-patching stress patches
    (KmcSimulation2D._precompute_patch_kernels) for the benchmark material on a
    16 x 12 grid, radius 3 and a radius whose window wraps the grid (9)."""
    import types
    from mgkmc import kmc_simulator as KS
    E, nu, _, _ = W.ls2d_problem(16, 12, seed=71)
    out = dict(E=E, nu=nu)
    for R in (3, 9):
        host = types.SimpleNamespace(patch_radius=R, nx=16, ny=12, nu_field=nu, pixel=1.0,
                                     plane_mode="plane_strain", solver_args={})
        KS.KmcSimulation2D._precompute_patch_kernels(host, E)
        out[f"kernels_r{R}"] = np.stack(host.patch_kernels)
        out[f"missing_r{R}"] = np.stack(host.patch_missing_mean)
    save("kmc2d_patch_16x12", **out)


def kmc2d_trajectory_fixtures():
    """A short trajectory of the reference's own KMC driver
    (KmcSimulation2D.run_simulation, kmc_simulator.py:796-1157): small-strain
    linear elasticity, KMC mode, softening off, every draw from numpy's global
    stream (select_event_2d replaced by its pure-Python body, whose uniform
    draw then comes from that stream instead of numba's).  Saves the initial
    catalog and barriers, the RandomState state the run starts from, the
    events (x, y, m, time) seen by the flip callback, the final macro strain,
    stress and eigenstrain fields."""
    import tempfile
    from mgkmc import kmc_simulator as KS
    nx, ny, M = 12, 8, 4
    rng = np.random.default_rng(41)
    E, nu = W.ls2d_material(nx, ny, rng)
    KS.select_event_2d = KF.select_event_2d.py_func
    np.random.seed(5)
    with tempfile.TemporaryDirectory() as tmp:
        sim = KS.KmcSimulation2D(nx, ny, M, 0.1, E, nu, barrier_generator="gaussian",
                                 barrier_kwargs=dict(mean=0.6, std=0.15, min_cutoff=0.3), softening_cap=2.0,
                                 jp=0.0, jt=0.0, temperature=300.0, strain_rate=1e7, output_dir=tmp)
        cat0, Q00 = sim.catalog.copy(), sim.Q0.copy()
        st = np.random.get_state()
        events = []
        sim.flip_callback = lambda s, x, y, m, *rest: events.append((x, y, m, s.time))
        sim.run_simulation(60, 1e-4, component=(0, 0), stress_targets={(1, 1): 0.0}, mixed_tol=1e4,
                           mixed_max_iter=50, enable_console_log=False, enable_summary_log=False,
                           enable_global_log=False)
    ev = np.array([e[:3] for e in events], dtype=np.int64).reshape(-1, 3)
    times = np.array([e[3] for e in events], dtype=np.float64)
    print(f"reference trajectory: {len(events)} events, final strain {sim.eps_macro[0, 0]:.5f}")
    save("kmc2d_traj_12x8", E=E, nu=nu, catalog0=cat0, Q00=Q00, rs_keys=st[1], rs_pos=np.int64(st[2]),
         rs_has_gauss=np.int64(st[3]), rs_gauss=np.float64(st[4]), n_steps=np.int64(60), step_size=1e-4,
         events=ev, times=times, eps_macro=sim.eps_macro, sig=sim.sig_field, eps_plastic=sim.eps_plastic,
         catalog=sim.catalog, Q0=sim.Q0)
    KS.select_event_2d = KF.select_event_2d


def driver_fixtures():
    """The reference's 3D mixed-BC small-strain ramp and its 3D finite-strain
    load ramp (Newton-CG, SVK), both run end to end."""
    rng = np.random.default_rng(13)
    shape = (8, 6, 4)
    E, nu = W.ls3d_material(*shape, rng)
    mask = np.ones((3, 3), bool)
    mask[1, 1] = mask[2, 2] = False
    target = np.zeros((3, 3))
    target[0, 0] = 0.01
    target[0, 1] = target[1, 0] = 0.002
    epsM, sigM, eps_l, sig_l = LES.linear_elastic_simulation_3d(
        E, nu, mask, target, n_steps=2, tol_ls=1e-10, max_iter_ls=300, tol_macro=1e3, max_iter_macro=30,
        enable_console=False)
    save("ls3d_macro_8x6x4", E=E, nu=nu, mask=mask, target=target, epsM=np.array(epsM), sigM=np.array(sigM),
         eps_last=eps_l[-1], sig_last=sig_l[-1])

    rng = np.random.default_rng(14)
    shape = (6, 6, 6)
    E, nu, _ = W.fs3d_material(*shape, rng)
    Fm, Sm, Pm, F_l, S_l = FS.finite_strain_simulation_3d(
        E, nu, (0, 0), 0.01, 2, mixed_targets={(1, 1): 0.0, (2, 2): 0.0}, tol_NW=1e-10, tol_CG=1e-11, max_NW=30,
        tol_macro=1e3, max_iter_macro=30, enable_console=False, model_type="svk", solver="newton_cg")
    save("fs3d_sim_6", E=E, nu=nu, F_macro=Fm, Sig_macro=Sm, P_macro=Pm, F_last=F_l[-1], Sig_last=S_l[-1])


def kmc3d_trajectory_fixtures():
    """A short trajectory of the reference's own 3D driver
    (ThermalSimulation.run_simulation, aqs.py:682-1201): small strain, KMC
    mode, softening off, draws from numpy's global stream (select_event
    replaced by its pure-Python body).  apply_flip_soa is wrapped to record
    each flip's (x, y, z, m, time)."""
    import tempfile
    from mgkmc import aqs as AQ
    nx, ny, nz, M = 6, 6, 4, 4
    rng = np.random.default_rng(42)
    E, nu = W.ls3d_material(nx, ny, nz, rng)
    flips = []
    orig_flip = AQ.apply_flip_soa

    def rec_flip(eps_p, _, soft, tl, cat, x, y, z, m, t, *rest):
        flips.append((x, y, z, m, t))
        return orig_flip(eps_p, _, soft, tl, cat, x, y, z, m, t, *rest)

    AQ.select_event = SK.select_event.py_func
    AQ.apply_flip_soa = rec_flip
    np.random.seed(6)
    with tempfile.TemporaryDirectory() as tmp:
        sim = AQ.ThermalSimulation(nx, ny, nz, M, 0.1, E, nu, barrier_generator="gaussian",
                                   barrier_kwargs=dict(mean=0.4, std=0.15, min_cutoff=0.2), softening_cap=2.0,
                                   jp=0.0, jt=0.0, temperature=300.0, strain_rate=1e7, output_dir=tmp)
        cat0, Q00 = sim.catalog.copy(), sim.Q0.copy()
        st = np.random.get_state()
        sim.run_simulation(60, 1e-4, component=(0, 0), stress_targets={(1, 1): 0.0, (2, 2): 0.0}, mixed_tol=1e4,
                           mixed_max_iter=50, checkpoint_interval=None, enable_console_log=False,
                           enable_summary_log=False, enable_global_log=False, enable_cascade_log=False,
                           enable_kmc_log=False)
    AQ.select_event = SK.select_event
    AQ.apply_flip_soa = orig_flip
    ev = np.array([f[:4] for f in flips], dtype=np.int64).reshape(-1, 4)
    times = np.array([f[4] for f in flips], dtype=np.float64)
    print(f"reference 3D trajectory: {len(flips)} events, final strain {sim.eps_macro[0, 0]:.5f}")
    save("kmc3d_traj_6x6x4", E=E, nu=nu, catalog0=cat0, Q00=Q00, rs_keys=st[1], rs_pos=np.int64(st[2]),
         rs_has_gauss=np.int64(st[3]), rs_gauss=np.float64(st[4]), n_steps=np.int64(60), step_size=1e-4,
         events=ev, times=times, eps_macro=sim.eps_macro, sig=sim.sig_field, eps_plastic=sim.eps_plastic,
         catalog=sim.catalog, Q0=sim.Q0)


def fs2d_step_fixtures():
    """The reference's 2D finite-strain path, plane strain:
    * its Newton-CG load step (finite_strain_solver_step_2d, solver="newton_cg",
      :2356-2572), SVK without F_p, F_bar fully prescribed (1.01, 0.996).  With
      F_p, or with the Neo-Hookean law, or with a stress-controlled component,
      its BiCGSTAB solves stall at small right-hand sides on this medium
      (info 150) and the Newton loop diverges, so those converged states are
      pinned through the law instead;
    * its constitutive law (constitutive_hyperelastic_2d :591-1087) with a
      plastic eigen-deformation field, SVK and Neo-Hookean: P and the Cauchy
      stress at a perturbed F."""
    rng = np.random.default_rng(71)
    nx, ny = 12, 8
    E, nu = W.ls2d_material(nx, ny, rng)
    I2, I4, I4rt, I4s, II = FS._make_identity_tensors_2d(nx, ny)
    Ghat4 = FS.build_ghat4_2d(nx, ny, float(nx), float(ny))
    C4 = FS.build_C4_2d(E, nu, I4s, II, plane_mode="plane_strain")
    Fp = np.einsum("ij,xy->ijxy", np.eye(2), np.ones((nx, ny)))
    sel = rng.random((nx, ny)) < 0.15
    G = rng.standard_normal((2, 2, nx, ny))
    S = 0.5 * (G + G.transpose(1, 0, 2, 3))
    S -= 0.5 * (S[0, 0] + S[1, 1]) * np.eye(2)[:, :, None, None]
    S /= np.sqrt(np.sum(S * S, axis=(0, 1)))
    Fp += 0.05 * S * sel
    F0 = np.einsum("ij,xy->ijxy", np.eye(2), np.ones((nx, ny)))
    Fb = np.diag([1.01, 0.996])
    F, P, Sig, _, Fbo = FS.finite_strain_solver_step_2d(
        F0, Fb, Ghat4, C4, I2, I4, I4rt, Fp=None, driving_component=(0, 0), E_avg=E.mean(), nu_avg=nu.mean(),
        tol_NW=1e-9, tol_CG=1e-10, max_NW=30, enable_console=False, model_type="svk", plane_mode="plane_strain",
        solver="newton_cg")
    out = dict(E=E, nu=nu, Fp=Fp, F_bar=Fb, svk_F=F, svk_P=P, svk_Sig=Sig)
    Fr = F0 + 0.02 * rng.standard_normal((2, 2, nx, ny))
    out["F_law"] = Fr
    for model in ("svk", "neo_hookean"):
        Pl, _, F33 = FS.constitutive_hyperelastic_2d(Fr, C4, I2, I4, I4rt, Fp=Fp, model_type=model,
                                                     plane_mode="plane_strain")
        out[f"{model}_P_law"] = Pl
        out[f"{model}_Sig_law"] = FS.cauchy_from_P(Pl, Fr, F33=F33)
    save("fs2d_step_12x8", **out)


def fs2d_sim_fixtures():
    """The reference's 2D finite-strain load ramp (finite_strain_simulation_2d,
    :2580-2851), SVK, Newton-CG, F_xx driven to 1.01 in 2 steps with F_yy held
    at 1 (no stress-controlled component: see fs2d_step_fixtures).  Newton
    tolerance 1e-7: each load step converges in three Newton iterations, the
    last step of size ~3e-10; a fourth iteration, which a tighter tolerance
    asks for, meets the stalled BiCGSTAB solve and its line search fails."""
    rng = np.random.default_rng(72)
    E, nu = W.ls2d_material(12, 8, rng)
    Fm, Sm, Pm, F_l, S_l = FS.finite_strain_simulation_2d(
        E, nu, (0, 0), 0.01, 2, mixed_targets={}, tol_NW=1e-7, tol_CG=1e-8, max_NW=30, enable_console=False,
        model_type="svk", solver="newton_cg")
    save("fs2d_sim_12x8", E=E, nu=nu, F_macro=Fm, Sig_macro=Sm, P_macro=Pm, F_last=F_l[-1], Sig_last=S_l[-1])


def fs2d_pstress_fixtures():
    """The reference's 2D plane-stress Newton-CG load step
    (finite_strain_solver_step_2d, plane_mode="plane_stress", :2356-2572;
    SVK law :1038-1049 with the plane-stress lambda of build_C4_2d and the
    Cauchy stress with F33, :1094-1115), F_bar prescribed (1.01, 0.997), SVK,
    without F_p ("nofp") and with F_p of amplitude 0.02 on 15 % of voxels
    ("fp").  Newton tolerance 1e-7: a tighter one reaches the stalled
    BiCGSTAB solve (see fs2d_sim_fixtures) and its line search fails."""
    rng = np.random.default_rng(73)
    nx, ny = 12, 8
    E, nu = W.ls2d_material(nx, ny, rng)
    I2, I4, I4rt, I4s, II = FS._make_identity_tensors_2d(nx, ny)
    Ghat4 = FS.build_ghat4_2d(nx, ny, float(nx), float(ny))
    C4 = FS.build_C4_2d(E, nu, I4s, II, plane_mode="plane_stress")
    Fp = np.einsum("ij,xy->ijxy", np.eye(2), np.ones((nx, ny)))
    sel = rng.random((nx, ny)) < 0.15
    G = rng.standard_normal((2, 2, nx, ny))
    S = 0.5 * (G + G.transpose(1, 0, 2, 3))
    S -= 0.5 * (S[0, 0] + S[1, 1]) * np.eye(2)[:, :, None, None]
    S /= np.sqrt(np.sum(S * S, axis=(0, 1)))
    Fp += 0.02 * S * sel
    F0 = np.einsum("ij,xy->ijxy", np.eye(2), np.ones((nx, ny)))
    Fb = np.diag([1.01, 0.997])
    out = dict(E=E, nu=nu, Fp=Fp, F_bar=Fb)
    for tag, fp in (("nofp", None), ("fp", Fp)):
        F, P, Sig, _, _ = FS.finite_strain_solver_step_2d(
            F0, Fb, Ghat4, C4, I2, I4, I4rt, Fp=fp, driving_component=(0, 0), E_avg=E.mean(), nu_avg=nu.mean(),
            tol_NW=1e-7, tol_CG=1e-8, max_NW=30, enable_console=False, model_type="svk", plane_mode="plane_stress",
            solver="newton_cg")
        out.update({f"{tag}_F": F, f"{tag}_P": P, f"{tag}_Sig": Sig})
    # the plane-stress laws (:591-1087) with F_p at a perturbed F: P and the
    # Cauchy stress with the law's F33, SVK and Neo-Hookean (its out-of-plane
    # stretch from the per-voxel Newton solve)
    Fr = F0 + 0.02 * rng.standard_normal((2, 2, nx, ny))
    out["F_law"] = Fr
    for model in ("svk", "neo_hookean"):
        Pl, _, F33 = FS.constitutive_hyperelastic_2d(Fr, C4, I2, I4, I4rt, Fp=Fp, model_type=model,
                                                     plane_mode="plane_stress")
        out[f"{model}_P_law"] = Pl
        out[f"{model}_F33_law"] = F33
        out[f"{model}_Sig_law"] = FS.cauchy_from_P(Pl, Fr, F33=F33)
    # the Neo-Hookean plane-stress Newton-CG step, F_bar prescribed, no F_p
    F, P, Sig, _, _ = FS.finite_strain_solver_step_2d(
        F0, Fb, Ghat4, C4, I2, I4, I4rt, Fp=None, driving_component=(0, 0), E_avg=E.mean(), nu_avg=nu.mean(),
        tol_NW=1e-7, tol_CG=1e-8, max_NW=30, enable_console=False, model_type="neo_hookean",
        plane_mode="plane_stress", solver="newton_cg")
    out.update(nh_F=F, nh_P=P, nh_Sig=Sig)
    save("fs2d_pstress_12x8", **out)


def ls3d_landau_fixtures():
    """The reference's 3D Landau law (stress_from_strain_landau_3d) without
    capping, with piecewise and with smooth capping, and its LS solver
    (spectral_solver_landau_3d, the basic scheme) on a heterogeneous medium
    with eigenstrains, with and without capping, and at fixed iteration
    counts."""
    from mgkmc import elasticity as ELA
    rng = np.random.default_rng(74)
    shape = (12, 8, 6)
    E, nu = W.ls3d_material(*shape, rng)
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    v1, v2, v3, g1, g2, g3, g4 = LANDAU_V
    kw = dict(v1=v1, v2=v2, v3=v3, g1=g1, g2=g2, g3=g3, g4=g4)
    e = rng.normal(0, 0.02, shape + (3, 3))
    e = 0.5 * (e + np.swapaxes(e, -1, -2))
    out = dict(lam=lam, mu=mu, v=np.array(LANDAU_V), strain=e)
    out["sig_plain"] = ELA.stress_from_strain_landau_3d(e, lam, mu, **kw)
    out["sig_piecewise"] = ELA.stress_from_strain_landau_3d(e, lam, mu, **kw, strain_capping_enabled=True,
                                                            strain_capping_limit=0.015)
    out["sig_smooth"] = ELA.stress_from_strain_landau_3d(e, lam, mu, **kw, strain_capping_enabled=True,
                                                         strain_capping_limit=0.015, strain_capping_type="smooth",
                                                         strain_capping_smooth_power=2.0)
    ep = W.pure_shear_eigenstrain_3d(*shape, rng, frac=0.1)
    eb = np.array([[0.008, 0.002, 0.0], [0.002, -0.003, 0.001], [0.0, 0.001, -0.002]])
    out.update(eps_plastic=ep, eps_bar=eb)
    for k in (1, 3):
        eps, sig, _, _ = LES.spectral_solver_landau_3d(lam, mu, **kw, eps_bar=eb, eps_plastic=ep, max_iter=k, tol=0.0)
        out.update({f"eps_it{k}": eps, f"sig_it{k}": sig})
    eps, sig, _, _ = LES.spectral_solver_landau_3d(lam, mu, **kw, eps_bar=eb, eps_plastic=ep, max_iter=400, tol=1e-12)
    out.update(eps_conv=eps, sig_conv=sig)
    eps, sig, _, _ = LES.spectral_solver_landau_3d(lam, mu, **kw, eps_bar=eb, eps_plastic=ep, max_iter=400, tol=1e-12,
                                                   strain_capping_enabled=True, strain_capping_limit=0.01,
                                                   strain_capping_type="smooth", strain_capping_smooth_power=2.0)
    out.update(eps_cap=eps, sig_cap=sig)
    save("ls3d_landau_12x8x6", **out)


def nl_ramp_fixtures():
    """The reference's nonlinear small-strain load ramps
    (linear_elastic_simulator.py:1353-2517: secant_elastic_simulation_2d/3d,
    rose_elastic_simulation_2d, landau_elastic_simulation_2d/3d) on
    heterogeneous media: three load steps of a driven xx strain with every
    other component stress-free, so each load step's macro loop iterates
    (the Landau ramps with their secant-slope correction)."""
    rng = np.random.default_rng(81)

    def lame(E, nu):
        return E * nu / ((1 + nu) * (1 - 2 * nu)), E / (2 * (1 + nu))

    lam2, mu2 = lame(*W.ls2d_material(16, 12, rng))
    lam3, mu3 = lame(*W.ls3d_material(12, 8, 6, rng))
    m2 = np.zeros((2, 2), dtype=bool)
    m2[0, 0] = True
    m3 = np.zeros((3, 3), dtype=bool)
    m3[0, 0] = True
    t2, t3 = np.zeros((2, 2)), np.zeros((3, 3))
    common = dict(n_steps=3, tol_ls=1e-11, max_iter_ls=600, tol_macro=1e3, max_iter_macro=30, store=True,
                  enable_console=False)
    out = dict(lam2=lam2, mu2=mu2, lam3=lam3, mu3=mu3, mask2=m2, mask3=m3, v=np.array(LANDAU_V))
    runs = (
        ("secant2d", 0.02, lambda t: LES.secant_elastic_simulation_2d(lam2, mu2, 0.3, 50.0, m2, t, **common)),
        ("rose2d", 0.02, lambda t: LES.rose_elastic_simulation_2d(lam2, mu2, 30.0, 0.1, m2, t, **common)),
        ("rose2d_pst", 0.02, lambda t: LES.rose_elastic_simulation_2d(lam2, mu2, 30.0, 0.1, m2, t, **common,
                                                                      plane_mode="plane_stress")),
        ("secant3d", 0.02, lambda t: LES.secant_elastic_simulation_3d(lam3, mu3, 0.3, 50.0, m3, t, **common)),
        ("landau2d", 0.01, lambda t: LES.landau_elastic_simulation_2d(lam2, mu2, *LANDAU_V, m2, t, **common)),
        ("landau3d", 0.01, lambda t: LES.landau_elastic_simulation_3d(lam3, mu3, *LANDAU_V, m3, t, **common)),
    )
    # the (E, nu) fields each ramp hands to its VTK writer on the "last"
    # schedule, recorded from the reference's own call
    seen = {}

    def record(fname, eps, sig, E, nu, pixel=1.0, **kw):
        seen["E"], seen["nu"] = np.array(E), np.array(nu)

    LES.export_to_vtk = record
    common.update(vtk_path=os.path.join(HERE, "_unused"), vtk_interval="last")
    for tag, exx, run in runs:
        t = (t2 if "2d" in tag else t3).copy()
        t[0, 0] = exx
        seen.clear()
        em, sm, el, sl = run(t)
        out.update({f"{tag}_target": t, f"{tag}_eps_mac": em, f"{tag}_sig_mac": sm, f"{tag}_eps": el[-1],
                    f"{tag}_sig": sl[-1], f"{tag}_vtk_E": seen["E"], f"{tag}_vtk_nu": seen["nu"]})
    save("nl_ramps", **out)


ALL = ("ls2d_fixtures", "ls3d_fixtures", "kmc2d_fixtures", "kmc3d_fixtures", "fs3d_fixtures", "ls2d_secant_fixtures",
       "ls2d_rose_fixtures", "kmc2d_cascade_fixtures", "kmc2d_patch_fixtures", "ls3d_secant_fixtures",
       "ls2d_landau_fixtures", "kmc2d_trajectory_fixtures", "driver_fixtures",
       "kmc3d_trajectory_fixtures", "fs2d_step_fixtures",
       "fs2d_sim_fixtures", "ls3d_landau_fixtures", "fs2d_pstress_fixtures",
       "ls2d_landau_pstress_fixtures", "vtk_fixtures", "nl_ramp_fixtures")


if __name__ == "__main__":
    # python make_golden.py [fixture function names]  (default: all)
    for name in (sys.argv[1:] or ALL):
        globals()[name]()

