"""numpy restatement of the de Geus finite-strain Newton-Krylov step in 3D (oracle).

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).

Follows mgkmc/finite_strain_simulator.py:
  * ``solver_step_3d``  -- finite_strain_solver_step_3d :2967-3168 with
    solver="newton_cg": macro mixed-BC loop (:3019, :3121-3166), Newton branch
    (:3046-3119) with the alpha-halving line search (:3088-3114);
  * ``build_bc_3d``     -- build_finite_strain_bc_3d :2852-2899;
  * ``cauchy``          -- cauchy_from_P_3d :1892-1904;
  * ``project``         -- _project_3d with build_ghat4_3d (:1121-1188):
    (G:A)_ij = (A xi)_i xi_j / |xi|^2 (the einsum 'ijkl,lk->ij' with
    Ghat_ijlm = delta_im xi_j xi_l / |xi|^2), zero at DC and on Nyquist planes;
  * ``constitutive``    -- constitutive_hyperelastic_3d :1647-1885 with F_p
    (:1848-1861).  SVK is the reference's 3D law (:1843-1846).  Neo-Hookean
    is restated in 3D from the reference's 2D plane-strain form (:686-720):
    S = mu I + (lam ln Je - mu) C^-1, tangent lam C^-1 x C^-1 + (mu - lam ln
    Je)(C^-1 o C^-1 + transpose), since the reference's 3D code silently
    computes SVK when asked for Neo-Hookean.
The tangent is applied matrix-free.  The reference's operator
trans2(K4 : trans2(dF)) (:3064-3066) depends on which K4 branch runs:
  * with F_p (:1849-1859):  S_ref dF^T + Fp^-1 Y Fe^T,
        Y = C_eff : sym(Fe^T dF Fp^-1),  S_ref = Fp^-1 S Fp^-T
    (the transpose of dP/dF[dF]);
  * without F_p (the "mandel" branch, :1863-1871):  dF S + Fe Y',
        Y' = C_eff : sym(Fe^T dF)  (dP/dF[dF] itself).
tests/test_oracle_fs.py checks both against the reference's own K4.

Fields here are spatial-first (nx, ny, nz, 3, 3); the reference API is
tensor-first (3, 3, nx, ny, nz) -- use ``to_tensor_first`` / ``to_spatial``.
"""
import numpy as np
import scipy.sparse.linalg as spla


def to_spatial(A):
    return np.ascontiguousarray(np.moveaxis(A, (0, 1), (-2, -1)))


def to_tensor_first(A):
    return np.ascontiguousarray(np.moveaxis(A, (-2, -1), (0, 1)))


def _tr(A):
    return np.swapaxes(A, -1, -2)


def lame_3d(E, nu):
    # build_C4_3d :1628-1640 -> C4[0,1,0,1] = mu, C4[0,0,1,1] = lam
    return E * nu / ((1 + nu) * (1 - 2 * nu)), E / (2 * (1 + nu))


def det3(A):
    return (A[..., 0, 0] * (A[..., 1, 1] * A[..., 2, 2] - A[..., 1, 2] * A[..., 2, 1])
            - A[..., 0, 1] * (A[..., 1, 0] * A[..., 2, 2] - A[..., 1, 2] * A[..., 2, 0])
            + A[..., 0, 2] * (A[..., 1, 0] * A[..., 2, 1] - A[..., 1, 1] * A[..., 2, 0]))


def plane_stress_nh_x(Fe, lam2, mu):
    """x = F33^2 of the plane-stress Neo-Hookean law (:631-684) on the
    embedded problem: lam_3d = 2 mu lam2 / (2 mu - lam2) from the
    plane-stress lambda, Je the in-plane det(Fe), Newton on
    mu x + lam_3d/2 ln x = mu - lam_3d ln Je from x = 1, at most 10 steps,
    until every voxel's step is below 1e-12 (the reference's loop)."""
    lam3 = (2.0 * mu * lam2) / np.maximum(1e-14, 2.0 * mu - lam2)
    Je = np.maximum(1e-14, det3(Fe))
    x = np.ones_like(Je)
    target = mu - lam3 * np.log(Je)
    for _ in range(10):
        f = mu * x + 0.5 * lam3 * np.log(x) - target
        dx = -f / (mu + 0.5 * lam3 / x)
        x = np.maximum(1e-10, x + dx)
        if np.max(np.abs(dx)) < 1e-12:
            break
    return x, lam3


def constitutive(F, lam, mu, Fpi, model="svk", has_fp=True, plane_stress=False):
    """(P, state) with state holding what the tangent needs.  plane_stress:
    the embedded 2D plane-stress laws (lam the plane-stress lambda); the
    state then also holds F33."""
    I = np.eye(3)
    Fe = F @ Fpi
    C = _tr(Fe) @ Fe
    l = lam[..., None, None]
    m = mu[..., None, None]
    if model == "neo_hookean" and plane_stress:
        # :631-684: S = mu I - mu x C^-1; tangent lam* C^-1 (x) C^-1 + mu x (C^-1 . C^-1)
        x, lam3 = plane_stress_nh_x(Fe, lam, mu)
        Ci = np.linalg.inv(C)
        S = m * I + (-mu * x)[..., None, None] * Ci
        c = mu * x
        lam_t = (2.0 * lam3 * c) / np.maximum(1e-14, lam3 + 2.0 * c)
        st = dict(Fe=Fe, Fpi=Fpi, model=model, Ci=Ci, c=c, F33=np.sqrt(np.maximum(1e-12, x)))
        st["Sref"] = Fpi @ S @ _tr(Fpi)
        st["lam"], st["mu"] = lam_t, mu
        st["has_fp"] = has_fp
        return Fe @ S @ _tr(Fpi), st
    if model == "svk":
        Eg = 0.5 * (C - I)
        S = l * np.trace(Eg, axis1=-2, axis2=-1)[..., None, None] * I + 2 * m * Eg
        st = dict(Fe=Fe, Fpi=Fpi, model=model)
    elif model == "neo_hookean":
        Je = np.maximum(1e-14, det3(Fe))
        lnJ = np.log(Je)
        Ci = np.linalg.inv(C)
        S = m * I + (l * lnJ[..., None, None] - m) * Ci
        st = dict(Fe=Fe, Fpi=Fpi, model=model, Ci=Ci, c=(mu - lam * lnJ))
    else:
        raise ValueError(model)
    st["Sref"] = Fpi @ S @ _tr(Fpi)
    st["lam"], st["mu"] = lam, mu
    st["has_fp"] = has_fp
    if plane_stress:
        st["F33"] = plane_stress_f33(F, lam, mu, Fpi)
    P = Fe @ S @ _tr(Fpi)
    return P, st


def kdf(d, st):
    """trans2(K4 : trans2(dF)) of the reference, matrix-free."""
    Fe, Fpi = st["Fe"], st["Fpi"]
    X = _tr(Fe) @ d @ Fpi
    l = st["lam"][..., None, None]
    if st["model"] == "svk":
        Y = l * np.trace(X, axis1=-2, axis2=-1)[..., None, None] * np.eye(3) + st["mu"][..., None, None] * (X + _tr(X))
    else:
        Ci = st["Ci"]
        Y = (l * np.trace(Ci @ X, axis1=-2, axis2=-1)[..., None, None] * Ci
             + st["c"][..., None, None] * (Ci @ (X + _tr(X)) @ Ci))
    out = st["Sref"] @ _tr(d) + Fpi @ Y @ _tr(Fe)
    return out if st["has_fp"] else _tr(out)


def project(A):
    """Ghat4 : A in Fourier space (build_ghat4_3d; _project_3d)."""
    nx, ny, nz = A.shape[:3]
    xi = np.meshgrid(np.fft.fftfreq(nx), np.fft.fftfreq(ny), np.fft.fftfreq(nz), indexing="ij")
    xi2 = xi[0] ** 2 + xi[1] ** 2 + xi[2] ** 2
    zero = xi2 == 0
    for a, n in enumerate((nx, ny, nz)):
        if n % 2 == 0:
            zero = zero | (xi[a] == -0.5)
    Ah = np.fft.fftn(A, axes=(0, 1, 2))
    v = sum(xi[l][..., None] * Ah[..., :, l] for l in range(3))  # (A xi)_i
    R = v[..., :, None] * np.stack(xi, -1)[..., None, :] / np.where(zero, 1.0, xi2)[..., None, None]
    R[zero] = 0
    return np.fft.ifftn(R, axes=(0, 1, 2)).real


def cauchy(P, F, F33=None):
    """cauchy_from_P_3d (:1892-1904); with F33, the 2D cauchy_from_P's
    J = det(F) F33 (:1094-1115)."""
    J = det3(F)
    if F33 is not None:
        J = J * F33
    J = np.where(np.abs(J) < 1e-14, 1e-14, J)
    return P @ _tr(F) / J[..., None, None]


def plane_stress_f33(F, lam, mu, Fpi):
    """Out-of-plane stretch of the 2D plane-stress SVK law (:1042-1049) on the
    embedded problem (plane axes x, z): E the in-plane Green-Lagrange strain
    of Fe = F Fp^-1, E33 = -(lam / (2 mu)) tr E, F33 = sqrt(max(1e-12,
    1 + 2 E33)); lam is the plane-stress lambda."""
    Fe = F @ Fpi
    C = _tr(Fe) @ Fe
    trE = 0.5 * (C[..., 0, 0] - 1.0) + 0.5 * (C[..., 2, 2] - 1.0)
    return np.sqrt(np.maximum(1e-12, 1.0 + 2.0 * (-(lam / (2.0 * mu)) * trE)))


def build_bc_3d(driving_component, eps, mixed_targets, F_bar_initial=None):
    """build_finite_strain_bc_3d :2852-2899."""
    F_bar = np.eye(3) if F_bar_initial is None else F_bar_initial.copy()
    F_mask = np.zeros((3, 3), bool)
    P_target = np.zeros((3, 3))
    P_mask = np.zeros((3, 3), bool)
    i_d, j_d = driving_component
    F_bar[i_d, j_d] = 1.0 + eps if i_d == j_d else eps
    F_mask[i_d, j_d] = True
    for a in range(3):
        for b in range(3):
            if a != b and (a, b) != (i_d, j_d):
                F_bar[a, b] = 0.0
                F_mask[a, b] = True
    for k in range(3):
        if k == i_d and i_d == j_d:
            continue
        if (k, k) in mixed_targets:
            P_target[k, k] = mixed_targets[(k, k)]
            P_mask[k, k] = True
        else:
            F_bar[k, k] = 1.0
            F_mask[k, k] = True
    return F_bar, F_mask, P_target, P_mask


def newton(F_start, F_bar, lam, mu, Fpi, tol_NW, tol_CG, max_NW, model="svk", krylov="bicgstab",
           return_stats=False, has_fp=True, plane_stress=False):
    """Newton branch of finite_strain_solver_step_3d (:3046-3119)."""
    shape = F_start.shape
    DbarF = np.broadcast_to(F_bar - F_start.mean(axis=(0, 1, 2)), shape)
    P, st = constitutive(F_start, lam, mu, Fpi, model, has_fp, plane_stress)
    cur = dict(st=st)
    A = spla.LinearOperator((F_start.size, F_start.size),
                            matvec=lambda v: project(kdf(v.reshape(shape), cur["st"])).ravel(), dtype=float)
    solve = spla.bicgstab if krylov == "bicgstab" else spla.cg
    F_curr = F_start.copy()
    nmv = 0
    for i in range(max_NW):
        rhs = -project(kdf(DbarF, cur["st"])).ravel() if i == 0 else -project(P).ravel()
        its = [0]
        dFm, _ = solve(A, rhs, rtol=tol_CG, maxiter=150, callback=lambda xk: its.__setitem__(0, its[0] + 1))
        nmv += its[0]
        dF = dFm.reshape(shape)
        dX = DbarF + dF if i == 0 else dF
        alpha = 1.0
        for _ in range(16):
            Ft = F_curr + alpha * dX
            Je = det3(Ft @ Fpi)
            if np.any(Je <= 1e-4) or np.any(np.isnan(Je)):
                alpha *= 0.5
                continue
            Pt, stt = constitutive(Ft, lam, mu, Fpi, model, has_fp, plane_stress)
            if np.any(np.isnan(Pt)):
                alpha *= 0.5
                continue
            F_curr, P = Ft, Pt
            cur["st"] = stt
            break
        else:
            raise ValueError("Newton-CG line search failed to find a valid step.")
        if np.linalg.norm(dFm) / (np.linalg.norm(F_curr) + 1e-20) < tol_NW and i > 0:
            if return_stats:
                return F_curr, P, dict(newton=i + 1, krylov=nmv, F33=cur["st"].get("F33"))
            return F_curr, P
    raise ValueError(f"Newton-CG inner solver did not converge within {max_NW} iterations.")


def solver_step_3d(F, F_bar, E, nu, Fp, driving_component=(0, 0), P_target=None, P_mask=None, E_avg=None,
                   nu_avg=None, tol_NW=1e-5, tol_CG=1e-6, max_NW=50, tol_macro=1e6, max_iter_macro=20,
                   model="svk", krylov="bicgstab", lame=None, plane_stress=False):
    """finite_strain_solver_step_3d (:2967-3168), Newton branch, spatial-first fields.
    Returns (F, P, Sig, F_bar_current).  ``lame`` = (lam, mu) fields replace
    the ones from (E, nu); ``plane_stress``: the embedded 2D plane-stress
    problem (SVK or Neo-Hookean; lam the plane-stress lambda), whose Cauchy
    stress carries F33."""
    lam, mu = lame_3d(E, nu) if lame is None else lame
    Fpi = np.linalg.inv(Fp) if Fp is not None else np.broadcast_to(np.eye(3), F.shape)
    E_avg = E.mean() if E_avg is None else E_avg
    nu_avg = nu.mean() if nu_avg is None else nu_avg
    P_target = np.zeros((3, 3)) if P_target is None else P_target
    P_mask = np.zeros((3, 3), bool) if P_mask is None else P_mask
    F_start = F.copy()
    F_bar_cur = F_bar.copy()
    i_d, j_d = driving_component
    upd = np.zeros((3, 3), bool)
    for a in range(3):
        if P_mask[a, a] and (a, a) != (i_d, j_d):
            upd[a, a] = True
    prev_F = prev_s = None
    max_err = 0.0
    for it in range(max_iter_macro):
        F_curr, P, stats = newton(F_start, F_bar_cur, lam, mu, Fpi, tol_NW, tol_CG, max_NW, model, krylov,
                                  return_stats=True, has_fp=Fp is not None, plane_stress=plane_stress)
        Sig = cauchy(P, F_curr, stats["F33"] if plane_stress else None)
        Sm = Sig.mean(axis=(0, 1, 2))
        if not np.any(P_mask):
            return F_curr, P, Sig, F_bar_cur
        err = np.zeros((3, 3))
        err[P_mask] = P_target[P_mask] - Sm[P_mask]
        max_err = np.max(np.abs(err[P_mask]))
        if max_err < tol_macro:
            return F_curr, P, Sig, F_bar_cur
        dFm = np.clip((err - nu_avg * np.trace(err) * np.eye(3)) / E_avg, -0.01, 0.01)
        d_sc = dFm[upd]
        Fb_sc = F_bar_cur[upd].copy()
        s_sc = Sm[upd].copy()
        if prev_F is not None:
            dh = Fb_sc - prev_F
            with np.errstate(divide="ignore", invalid="ignore"):
                slope = (s_sc - prev_s) / dh
            e_sc = err[upd]
            ok = np.isfinite(slope) & (np.abs(dh) > 1e-14) & (slope > 0.01 * E_avg)
            d_sc[ok] = np.clip(e_sc[ok] / slope[ok], -0.01, 0.01)
        prev_F, prev_s = Fb_sc, s_sc
        F_bar_cur[upd] += d_sc
        F_start = F_curr
    raise ValueError(f"Outer BC loop did not converge after {max_iter_macro} iterations. "
                     f"Final max stress error: {max_err:.2e} Pa")


def constitutive_2d_plane_strain_nh(F2, lam, mu):
    """2D plane-strain Neo-Hookean P (finite_strain_simulator.py:686-720), for pinning the 3D restatement."""
    F3 = np.zeros(F2.shape[:-2] + (3, 3))
    F3[..., :2, :2] = F2
    F3[..., 2, 2] = 1.0
    P, st = constitutive(F3, lam, mu, np.broadcast_to(np.eye(3), F3.shape), "neo_hookean", has_fp=False)
    return P[..., :2, :2], st


# 2D plane strain as a 3D problem: the plane's axes (x, y) become the 3D axes
# (x, z), the out-of-plane axis is the 3D y axis (one voxel thick) with
# F_yy = 1.  Tensor indices map 0 -> 0, 1 -> 2.
PLANE_AXES = (0, 2)


def embed_plane_2d(A2, fill=1.0):
    """Tensor-first (2,2,nx,ny) -> spatial-first (nx,1,ny,3,3); the
    out-of-plane diagonal entry is ``fill`` (1 for F and F_p, 0 for P)."""
    nx, ny = A2.shape[2:]
    A3 = np.zeros((nx, 1, ny, 3, 3))
    for a, i in enumerate(PLANE_AXES):
        for b, j in enumerate(PLANE_AXES):
            A3[:, 0, :, i, j] = A2[a, b]
    A3[:, 0, :, 1, 1] = fill
    return A3


def extract_plane_2d(A3):
    """Spatial-first (nx,1,ny,3,3) -> tensor-first (2,2,nx,ny)."""
    nx, _, ny = A3.shape[:3]
    A2 = np.zeros((2, 2, nx, ny))
    for a, i in enumerate(PLANE_AXES):
        for b, j in enumerate(PLANE_AXES):
            A2[a, b] = A3[:, 0, :, i, j]
    return A2
