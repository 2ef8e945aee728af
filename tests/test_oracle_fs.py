"""The finite-strain oracle (oracle/fs.py) reproduces the unmodified
reference: constitutive P, the matrix-free tangent operator, the projection,
one mixed-BC Newton-Krylov load step (golden fixture), and the 2D
plane-strain Neo-Hookean law the 3D Neo-Hookean is restated from."""
import numpy as np
import pytest

from oracle import fs as OF


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def test_constitutive_tangent_projection(golden):
    g = golden("fs3d_svk_6")
    lam, mu = OF.lame_3d(g["E"], g["nu"])
    F = OF.to_spatial(g["F_trial"])
    Fpi = np.linalg.inv(OF.to_spatial(g["Fp"]))
    P, st = OF.constitutive(F, lam, mu, Fpi, "svk")
    assert rel(OF.to_tensor_first(P), g["P_trial"]) < 1e-13
    KdF = OF.kdf(OF.to_spatial(g["dF"]), st)
    assert rel(OF.to_tensor_first(KdF), g["KdF"]) < 1e-13
    GK = OF.project(KdF)
    assert rel(OF.to_tensor_first(GK), g["GKdF"]) < 1e-12


def test_newton_step_matches_reference(golden):
    g = golden("fs3d_svk_6")
    F0 = OF.to_spatial(np.einsum("ij,xyz->ijxyz", np.eye(3), np.ones(g["E"].shape)))
    F, P, Sig, Fb = OF.solver_step_3d(F0, g["F_bar_in"], g["E"], g["nu"], OF.to_spatial(g["Fp"]), (0, 0),
                                      np.zeros((3, 3)), g["P_mask"], tol_NW=1e-10, tol_CG=1e-10, max_NW=30,
                                      tol_macro=1e3, max_iter_macro=30, model="svk", krylov="bicgstab")
    assert rel(OF.to_tensor_first(F), g["F"]) < 1e-9
    assert rel(OF.to_tensor_first(P), g["P"]) < 1e-9
    assert rel(OF.to_tensor_first(Sig), g["Sig"]) < 1e-9
    assert np.max(np.abs(Fb - g["F_bar_out"])) < 1e-9
    # CG instead of BiCGSTAB converges to the same load-step solution
    F2, P2, _, _ = OF.solver_step_3d(F0, g["F_bar_in"], g["E"], g["nu"], OF.to_spatial(g["Fp"]), (0, 0),
                                     np.zeros((3, 3)), g["P_mask"], tol_NW=1e-10, tol_CG=1e-10, max_NW=30,
                                     tol_macro=1e3, max_iter_macro=30, model="svk", krylov="cg")
    assert rel(OF.to_tensor_first(F2), g["F"]) < 1e-9


def test_neo_hookean_2d_plane_strain(golden):
    g = golden("fs2d_neohookean_5")
    lam, mu = OF.lame_3d(g["E"], g["nu"])  # plane strain: the 3D Lame constants (build_C4_2d)
    F2 = OF.to_spatial(g["F"])
    P, st = OF.constitutive_2d_plane_strain_nh(F2, lam, mu)
    assert rel(OF.to_tensor_first(P), g["P"]) < 1e-13
    # in-plane tangent: the reference K4 (no F_p, mandel branch) against ours
    rng = np.random.default_rng(0)
    d2 = rng.standard_normal(F2.shape)
    ref = np.einsum("ijxy->jixy", np.einsum("ijklxy,lkxy->ijxy", g["K4"], np.einsum("ijxy->jixy", OF.to_tensor_first(d2))))
    d3 = np.zeros(d2.shape[:-2] + (3, 3)); d3[..., :2, :2] = d2
    ours = OF.kdf(d3, st)[..., :2, :2]
    assert rel(OF.to_tensor_first(ours), ref) < 1e-12


def test_neo_hookean_close_to_svk_at_small_strain():
    # the reference's tests/test_finite_strain_kmc.py:127-169 check in 2D, here in 3D
    from mgkmc_b200 import workloads as W
    rng = np.random.default_rng(4)
    E, nu, Fp = W.fs3d_material(6, 6, 6, rng, fp_frac=0.0)
    F0 = np.broadcast_to(np.eye(3), (6, 6, 6, 3, 3)).copy()
    Fb, Fm, Pt, Pm = OF.build_bc_3d((0, 0), 1e-5, {(1, 1): 0.0, (2, 2): 0.0})
    out = {}
    for model in ("svk", "neo_hookean"):
        F, P, Sig, _ = OF.solver_step_3d(F0, Fb, E, nu, None, (0, 0), Pt, Pm, tol_NW=1e-10, tol_CG=1e-10,
                                         max_NW=30, tol_macro=1.0, max_iter_macro=30, model=model, krylov="cg")
        out[model] = Sig.mean(axis=(0, 1, 2))
    assert abs(out["svk"][0, 0] - out["neo_hookean"][0, 0]) < 1e-3 * abs(out["svk"][0, 0])


@pytest.mark.parametrize("model", ["svk", "neo_hookean"])
def test_plane_strain_law_embedded_in_3d(golden, model):
    # the reference's 2D plane-strain law (constitutive_hyperelastic_2d,
    # :591-1087) with F_p equals the 3D law on the embedded problem (out-of-
    # plane axis y, F_yy = 1): P and the Cauchy stress
    g = golden("fs2d_step_12x8")
    nx, ny = g["E"].shape
    lam, mu = OF.lame_3d(g["E"][:, None, :], g["nu"][:, None, :])
    F3 = OF.embed_plane_2d(g["F_law"])
    Fpi = np.linalg.inv(OF.embed_plane_2d(g["Fp"]))
    P3, _ = OF.constitutive(F3, lam, mu, Fpi, model, has_fp=True)
    P2 = OF.extract_plane_2d(P3)
    ref = g[f"{model}_P_law"]
    assert np.max(np.abs(P2 - ref)) < 1e-12 * np.max(np.abs(ref))
    S2 = OF.extract_plane_2d(OF.cauchy(P3, F3))
    assert np.max(np.abs(S2 - g[f"{model}_Sig_law"])) < 1e-12 * np.max(np.abs(ref))


def test_plane_strain_newton_step_embedded_in_3d(golden):
    # the reference's 2D Newton-CG step (SVK, F_bar prescribed) equals the 3D
    # oracle step on the embedded problem
    g = golden("fs2d_step_12x8")
    nx, ny = g["E"].shape
    E3, nu3 = g["E"][:, None, :], g["nu"][:, None, :]
    F0 = OF.embed_plane_2d(np.einsum("ij,xy->ijxy", np.eye(2), np.ones((nx, ny))))
    Fb = np.eye(3)
    Fb[0, 0], Fb[2, 2] = g["F_bar"][0, 0], g["F_bar"][1, 1]
    F, P, Sig, _ = OF.solver_step_3d(F0, Fb, E3, nu3, None, (0, 0), None, None, tol_NW=1e-12, tol_CG=1e-13,
                                     max_NW=30, model="svk", krylov="cg")
    assert np.max(np.abs(OF.extract_plane_2d(F) - g["svk_F"])) < 1e-9
    assert np.max(np.abs(OF.extract_plane_2d(P) - g["svk_P"])) < 1e-9 * np.max(np.abs(g["svk_P"]))


def _pstress_oracle(g, fp):
    E, nu = g["E"], g["nu"]
    nx, ny = E.shape
    lam, mu = E * nu / (1.0 - nu ** 2), E / (2 * (1 + nu))  # build_C4_2d, plane stress
    F0 = OF.embed_plane_2d(np.einsum("ij,xy->ijxy", np.eye(2), np.ones((nx, ny))))
    Fb = np.eye(3)
    Fb[0, 0], Fb[2, 2] = g["F_bar"][0, 0], g["F_bar"][1, 1]
    return OF.solver_step_3d(F0, Fb, E[:, None, :], nu[:, None, :], None if fp is None else OF.embed_plane_2d(fp),
                             (0, 0), None, None, tol_NW=1e-12, tol_CG=1e-13, max_NW=40, model="svk", krylov="cg",
                             lame=(lam[:, None, :], mu[:, None, :]), plane_stress=True)


def test_plane_stress_newton_step_embedded_in_3d(golden):
    # the reference's 2D plane-stress Newton-CG step (SVK, F_bar prescribed)
    # equals the oracle's step on the embedded problem with the plane-stress
    # lambda and the Cauchy stress divided by det(F) F33
    g = golden("fs2d_pstress_12x8")
    F, P, Sig, _ = _pstress_oracle(g, None)
    assert np.max(np.abs(OF.extract_plane_2d(F) - g["nofp_F"])) < 1e-9
    for a, b in ((P, g["nofp_P"]), (Sig, g["nofp_Sig"])):
        assert np.max(np.abs(OF.extract_plane_2d(a) - b)) < 1e-9 * np.max(np.abs(b))


def test_plane_stress_newton_step_with_fp_embedded_in_3d(golden):
    # with F_p the reference's step stops at Newton tolerance 1e-7 (a tighter
    # one reaches its stalled BiCGSTAB solve): its equilibrium residual
    # |G:P| / |P| is ~3e-8, and the fields agree to that level; the oracle's
    # own residual is below 1e-11
    g = golden("fs2d_pstress_12x8")
    F, P, Sig, _ = _pstress_oracle(g, g["Fp"])
    res = lambda P3: np.linalg.norm(OF.project(P3)) / np.linalg.norm(P3)
    assert res(P) < 1e-11
    ref_res = res(OF.embed_plane_2d(g["fp_P"], 0.0))
    assert 1e-9 < ref_res < 1e-7
    assert np.max(np.abs(OF.extract_plane_2d(F) - g["fp_F"])) < 1e-8
    for a, b in ((P, g["fp_P"]), (Sig, g["fp_Sig"])):
        assert np.max(np.abs(OF.extract_plane_2d(a) - b)) < 2e-7 * np.max(np.abs(b))


@pytest.mark.parametrize("model", ["svk", "neo_hookean"])
def test_plane_stress_law_embedded_in_3d(golden, model):
    # the reference's 2D plane-stress laws with F_p (:591-1087; Neo-Hookean
    # with its out-of-plane Newton solve) equal the oracle's on the embedded
    # problem with the plane-stress lambda: P, F33 and the Cauchy stress
    g = golden("fs2d_pstress_12x8")
    E, nu = g["E"], g["nu"]
    lam, mu = (E * nu / (1.0 - nu ** 2))[:, None, :], (E / (2 * (1 + nu)))[:, None, :]
    F3 = OF.embed_plane_2d(g["F_law"])
    Fpi = np.linalg.inv(OF.embed_plane_2d(g["Fp"]))
    P3, st = OF.constitutive(F3, lam, mu, Fpi, model, has_fp=True, plane_stress=True)
    ref = g[f"{model}_P_law"]
    assert np.max(np.abs(OF.extract_plane_2d(P3) - ref)) < 1e-12 * np.max(np.abs(ref))
    assert np.max(np.abs(st["F33"][:, 0, :] - g[f"{model}_F33_law"])) < 1e-14
    S2 = OF.extract_plane_2d(OF.cauchy(P3, F3, st["F33"]))
    assert np.max(np.abs(S2 - g[f"{model}_Sig_law"])) < 1e-12 * np.max(np.abs(ref))


def test_plane_stress_neo_hookean_step_embedded_in_3d(golden):
    # the reference's plane-stress Neo-Hookean Newton-CG step (F_bar
    # prescribed, no F_p) equals the oracle's step on the embedded problem
    g = golden("fs2d_pstress_12x8")
    E, nu = g["E"], g["nu"]
    nx, ny = E.shape
    lam, mu = E * nu / (1.0 - nu ** 2), E / (2 * (1 + nu))
    F0 = OF.embed_plane_2d(np.einsum("ij,xy->ijxy", np.eye(2), np.ones((nx, ny))))
    Fb = np.eye(3)
    Fb[0, 0], Fb[2, 2] = g["F_bar"][0, 0], g["F_bar"][1, 1]
    F, P, Sig, _ = OF.solver_step_3d(F0, Fb, E[:, None, :], nu[:, None, :], None, (0, 0), None, None, tol_NW=1e-12,
                                     tol_CG=1e-13, max_NW=40, model="neo_hookean", krylov="cg",
                                     lame=(lam[:, None, :], mu[:, None, :]), plane_stress=True)
    assert np.max(np.abs(OF.extract_plane_2d(F) - g["nh_F"])) < 1e-9
    for a, b in ((P, g["nh_P"]), (Sig, g["nh_Sig"])):
        assert np.max(np.abs(OF.extract_plane_2d(a) - b)) < 1e-9 * np.max(np.abs(b))
