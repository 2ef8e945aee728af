"""numpy restatement of the small-strain Lippmann-Schwinger solver (oracle).

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).

Follows mgkmc/linear_elastic_simulator.py:
  * ``spectral_solver_2d``  -- :12-88
  * ``spectral_solver_3d``  -- :274-376
  * ``spectral_solver_secant_2d`` -- :614-765 (secant degradation law,
    elasticity.py:112-150, :189-260)
  * ``spectral_solver_rose_2d`` -- :852-950 (Rose law, elasticity.py:868-944)
  * ``mixed_bc_solve_2d``   -- the macro mixed stress/strain loop of
    ``linear_elastic_simulation_2d`` :176-197 with the compliance correction of
    :150-152, here with an eigenstrain field (the reference driver has no
    ``eps_plastic`` argument, so the benchmark harness restates the loop).
and mgkmc/elasticity.py:3-105 for the Lame constants, Hooke's law and the
isotropic Green operator.  FFTs are ortho-normalised complex fftn/ifftn with
``.real`` taken on the inverse (mgkmc/fft.py:22-31).
"""
import numpy as np


def lame_2d(E, nu, plane_mode="plane_strain"):
    # mgkmc/elasticity.py:3-10
    mu = E / (2 * (1 + nu))
    if plane_mode == "plane_stress":
        lam = E * nu / (1 - nu ** 2)
    else:
        lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    return lam, mu


def lame_3d(E, nu):
    # mgkmc/elasticity.py:55-59
    mu = E / (2 * (1 + nu))
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    return lam, mu


def hooke(eps, lam, mu, d):
    # mgkmc/elasticity.py:12-18 and :62-67: sigma = 2 mu eps + lam tr(eps) I
    tr = np.trace(eps, axis1=-2, axis2=-1)[..., None, None]
    I = np.eye(d)
    return 2 * np.asarray(mu)[..., None, None] * eps + np.asarray(lam)[..., None, None] * tr * I


def wave_vectors(shape, pixel=1.0):
    # mgkmc/fft.py:9-20
    ks = [2 * np.pi * np.fft.fftfreq(n, d=(n * pixel) / n) for n in shape]
    return np.meshgrid(*ks, indexing="ij")


def green_operator(q, lam0, mu0):
    """Gamma^0_khij(q), spatial axes first (mgkmc/elasticity.py:20-53, :70-105)."""
    d = len(q)
    k2 = sum(qi * qi for qi in q)
    k2s = k2.copy()
    k2s[(0,) * d] = 1.0
    A = 1.0 / (4 * mu0)
    B = (lam0 + mu0) / (mu0 * (lam0 + 2 * mu0))
    G = np.zeros(q[0].shape + (d, d, d, d))
    for k in range(d):
        for h in range(d):
            for i in range(d):
                for j in range(d):
                    t1 = 0.0
                    if k == i:
                        t1 = t1 + q[h] * q[j]
                    if h == i:
                        t1 = t1 + q[k] * q[j]
                    if k == j:
                        t1 = t1 + q[h] * q[i]
                    if h == j:
                        t1 = t1 + q[k] * q[i]
                    G[..., k, h, i, j] = A * t1 / k2s - B * (q[k] * q[h] * q[i] * q[j]) / (k2s * k2s)
    G[(0,) * d] = 0
    return G


def spectral_solver(E, nu, eps_bar, eps_plastic=None, max_iter=200, tol=1e-6,
                    pixel=1.0, plane_mode="plane_strain", eps_init=None,
                    return_info=False):
    """LS fixed point in 2D or 3D (dimension from E.ndim).

    Returns (eps, sig, eps_mean, sig_mean) like the reference, plus
    (iterations, last diff) when ``return_info``.
    """
    d = E.ndim
    axes = tuple(range(d))
    E_avg = E.mean()
    nu_avg = nu.mean()
    if d == 2:
        lam, mu = lame_2d(E, nu, plane_mode)
        lam0, mu0 = lame_2d(E_avg, nu_avg, plane_mode)
    else:
        lam, mu = lame_3d(E, nu)
        lam0, mu0 = lame_3d(E_avg, nu_avg)
    G = green_operator(wave_vectors(E.shape, pixel), lam0, mu0)
    # initial field (linear_elastic_simulator.py:32-41)
    if eps_init is not None:
        eps = eps_init.copy()
        eps += eps_bar - eps_init.mean(axis=axes)
    else:
        eps = np.broadcast_to(eps_bar, E.shape + (d, d)).copy()
    ep = eps_plastic
    it_done = 0
    diff = np.inf
    sub = "xyz"[:d]
    for it in range(max_iter):
        sig = hooke(eps - ep if ep is not None else eps, lam, mu, d)
        sig0 = hooke(eps, lam0, mu0, d)
        tau = sig - sig0
        tau_hat = np.fft.fftn(tau, axes=axes, norm="ortho")
        et_hat = -np.einsum(f"{sub}khij,{sub}ij->{sub}kh", G, tau_hat)
        et = np.fft.ifftn(et_hat, axes=axes, norm="ortho").real
        et -= et.mean(axis=axes)
        eps_new = eps_bar + et
        diff = np.linalg.norm(eps_new - eps) / (np.linalg.norm(eps) + 1e-20)
        eps = eps_new
        it_done = it + 1
        if diff < tol:
            break
    sig_out = hooke(eps - ep if ep is not None else eps, lam, mu, d)
    out = (eps, sig_out, eps.mean(axis=axes), sig_out.mean(axis=axes))
    if return_info:
        return out + (it_done, diff)
    return out


def von_mises_strain_2d(e):
    """sqrt(2/3 e':e'), plane strain (e'_33 = -(e11 + e22)/3)
    (mgkmc/elasticity.py:112-150)."""
    e11, e22, e12, e21 = e[..., 0, 0], e[..., 1, 1], e[..., 0, 1], e[..., 1, 0]
    tr3 = (e11 + e22) / 3.0
    return np.sqrt((2.0 / 3.0) * ((e11 - tr3) ** 2 + (e22 - tr3) ** 2 + (-(e11 + e22) / 3.0) ** 2
                                  + 0.5 * (e12 + e21) ** 2))


def secant_stress_2d(e, lam, mu, d, k):
    """lam tr(e) I + 2 mu (1 - d (1 - exp(-k eq(e)))) e
    (mgkmc/elasticity.py:189-260)."""
    mu_sec = mu * (1.0 - d * (1.0 - np.exp(-k * von_mises_strain_2d(e))))
    return hooke(e, lam, mu_sec, 2)


def spectral_solver_secant_2d(lam, mu, d, k, eps_bar, eps_plastic=None, max_iter=400, tol=1e-6, pixel=1.0,
                              eps_init=None, return_info=False):
    """Secant-degradation LS fixed point (mgkmc/linear_elastic_simulator.py:
    614-765): reference medium (mean lam, mean mu) fixed; tau = sigma_sec(eps
    - eps_p) - C0:eps; same Green step, update and stopping rule as the linear
    solver."""
    lam0, mu0 = float(np.mean(lam)), float(np.mean(mu))
    shape = np.shape(lam)
    axes = (0, 1)
    G = green_operator(wave_vectors(shape, pixel), lam0, mu0)
    if eps_init is not None:
        eps = eps_init.copy()
        eps += eps_bar - eps_init.mean(axis=axes)
    else:
        eps = np.broadcast_to(eps_bar, shape + (2, 2)).copy()
    ep = eps_plastic
    it_done, diff = 0, np.inf
    for it in range(max_iter):
        sig = secant_stress_2d(eps - ep if ep is not None else eps, lam, mu, d, k)
        tau = sig - hooke(eps, lam0, mu0, 2)
        tau_hat = np.fft.fftn(tau, axes=axes, norm="ortho")
        et = np.fft.ifftn(-np.einsum("xykhij,xyij->xykh", G, tau_hat), axes=axes, norm="ortho").real
        et -= et.mean(axis=axes)
        eps_new = eps_bar + et
        diff = np.linalg.norm(eps_new - eps) / (np.linalg.norm(eps) + 1e-20)
        eps = eps_new
        it_done = it + 1
        if diff < tol:
            break
    sig_out = secant_stress_2d(eps - ep if ep is not None else eps, lam, mu, d, k)
    out = (eps, sig_out, eps.mean(axis=axes), sig_out.mean(axis=axes))
    return out + (it_done, diff) if return_info else out


def von_mises_strain_3d(e):
    """sqrt(2/3 e':e') (mgkmc/elasticity.py:665-700)."""
    tr3 = (e[..., 0, 0] + e[..., 1, 1] + e[..., 2, 2]) / 3.0
    return np.sqrt((2.0 / 3.0) * ((e[..., 0, 0] - tr3) ** 2 + (e[..., 1, 1] - tr3) ** 2
                                  + (e[..., 2, 2] - tr3) ** 2
                                  + 0.5 * ((e[..., 0, 1] + e[..., 1, 0]) ** 2 + (e[..., 0, 2] + e[..., 2, 0]) ** 2
                                           + (e[..., 1, 2] + e[..., 2, 1]) ** 2)))


def secant_stress_3d(e, lam, mu, d, k):
    """lam tr(e) I + 2 mu (1 - d (1 - exp(-k eq(e)))) e
    (mgkmc/elasticity.py:261-295, :703-728)."""
    mu_sec = mu * (1.0 - d * (1.0 - np.exp(-k * von_mises_strain_3d(e))))
    return hooke(e, lam, mu_sec, 3)


def spectral_solver_secant_3d(lam, mu, d, k, eps_bar, eps_plastic=None, max_iter=400, tol=1e-6, pixel=1.0,
                              eps_init=None, return_info=False):
    """Secant-degradation LS fixed point in 3D (mgkmc/linear_elastic_simulator.py:
    768-850): reference medium (mean lam, mean mu) fixed; tau = sigma_sec(eps
    - eps_p) - C0:eps; the linear solver's Green step, update and stopping
    rule."""
    lam0, mu0 = float(np.mean(lam)), float(np.mean(mu))
    shape = np.shape(lam)
    axes = (0, 1, 2)
    G = green_operator(wave_vectors(shape, pixel), lam0, mu0)
    if eps_init is not None:
        eps = eps_init.copy()
        eps += eps_bar - eps_init.mean(axis=axes)
    else:
        eps = np.broadcast_to(eps_bar, shape + (3, 3)).copy()
    ep = eps_plastic
    it_done, diff = 0, np.inf
    for it in range(max_iter):
        sig = secant_stress_3d(eps - ep if ep is not None else eps, lam, mu, d, k)
        tau = sig - hooke(eps, lam0, mu0, 3)
        tau_hat = np.fft.fftn(tau, axes=axes, norm="ortho")
        et = np.fft.ifftn(-np.einsum("xyzkhij,xyzij->xyzkh", G, tau_hat), axes=axes, norm="ortho").real
        et -= et.mean(axis=axes)
        eps_new = eps_bar + et
        diff = np.linalg.norm(eps_new - eps) / (np.linalg.norm(eps) + 1e-20)
        eps = eps_new
        it_done = it + 1
        if diff < tol:
            break
    sig_out = secant_stress_3d(eps - ep if ep is not None else eps, lam, mu, d, k)
    out = (eps, sig_out, eps.mean(axis=axes), sig_out.mean(axis=axes))
    return out + (it_done, diff) if return_info else out


def _landau_scalars_2d(a11, a22, a12, a21, e33, lam, mu, v, cap):
    """Capped components, invariants and Landau coefficients of the
    block-diagonal strain (in-plane a, out-of-plane e33)
    (mgkmc/elasticity.py:527-569).  cap: None or (type, E_cap, power)."""
    v1, v2, v3, g1, g2, g3, g4 = v
    m3 = (a11 + a22 + e33) / 3.0
    d11, d22, d33 = a11 - m3, a22 - m3, e33 - m3
    if cap is not None:
        cap_type, E_cap, cap_power = cap
        E_eq = np.sqrt(np.maximum(0.0, (2.0 / 3.0) * (d11 * d11 + d22 * d22 + d33 * d33 + 2.0 * a12 * a21)))
        f = np.ones_like(E_eq)
        nz = E_eq > 1e-12
        if cap_type == "smooth":
            rp = np.minimum(100.0, (E_eq[nz] / E_cap) ** cap_power)
            f[nz] = (E_cap / E_eq[nz]) * np.tanh(rp) ** (1.0 / cap_power)
            w = np.tanh(np.minimum(100.0, (E_eq / E_cap) ** cap_power)) ** 2
        else:
            capped = E_eq > E_cap
            np.divide(E_cap, E_eq, out=f, where=capped)
            w = capped.astype(float)
        c11, c22, c12, c21, c33 = f * d11 + m3, f * d22 + m3, f * a12, f * a21, f * d33 + m3
    else:
        w = None
        c11, c22, c12, c21, c33 = a11, a22, a12, a21, e33
    I1 = c11 + c22 + c33
    cross = c12 * c21
    tr2 = c11 * c11 + c22 * c22 + 2.0 * cross
    I2 = tr2 + c33 * c33
    t_ip = c11 + c22
    I3 = t_ip * (tr2 - (c11 * c22 - cross)) + c33 ** 3
    cI = lam * I1 + 0.5 * v1 * I1 ** 2 + v2 * I2 + (1.0 / 6.0) * g1 * I1 ** 3 + g2 * I1 * I2 + (4.0 / 3.0) * g3 * I3
    ce = 2.0 * (mu + v2 * I1 + 0.5 * g2 * I1 ** 2 + g4 * I2)
    ce2 = 4.0 * (v3 + g3 * I1)
    return I1, I2, c11, c22, c12, c21, c33, w, cI, ce, ce2


def landau_stress_2d(e, lam, mu, v, cap_type=None, cap_limit=None, cap_ratio=0.1, cap_power=1.0,
                     plane_stress=False, e33_state=None):
    """Landau small-strain stress (mgkmc/elasticity.py:487-639): v = (v1, v2,
    v3, g1, g2, g3, g4).  With cap_type "piecewise" or "smooth" the strain is
    capped at the equivalent strain E_cap (cap_limit, or sqrt(0.2 mean(mu) /
    |g4|) when it is None or <= 0 and g4 < 0, else 999) and a tangent
    2 cap_ratio mu w (e - e_capped) is added.  Plane strain: e33 = 0.  Plane
    stress (:571-616): e33 from Newton steps on sigma33 = 0 from the warm
    state (e33_state["e33"]) or the linear guess -lam/(lam + 2 mu) tr e, at
    most 20, until every voxel's step is below 1e-9; the stress is that of
    the last state evaluated before the final step; e33_state receives the
    stepped e33."""
    v1, v2, v3, g1, g2, g3, g4 = v
    a11, a22, a12, a21 = e[..., 0, 0], e[..., 1, 1], e[..., 0, 1], e[..., 1, 0]
    cap = None
    if cap_type is not None:
        mu_mean = np.mean(mu)
        E_cap = cap_limit if cap_limit is not None and cap_limit > 0 else (
            np.sqrt(0.2 * mu_mean / abs(g4)) if g4 < 0 else 999.0)
        cap = (cap_type, E_cap, cap_power)
        Gt = cap_ratio * mu
    if plane_stress:
        warm = None if e33_state is None else e33_state.get("e33")
        if warm is not None and warm.shape == a11.shape:
            e33 = warm.copy()
        else:
            e33 = -lam / (lam + 2.0 * mu) * (a11 + a22)
        for _ in range(20):
            I1, I2, c11, c22, c12, c21, c33, w, cI, ce, ce2 = _landau_scalars_2d(a11, a22, a12, a21, e33, lam, mu,
                                                                                   v, cap)
            s33 = cI + ce * c33 + ce2 * c33 ** 2
            dcI = lam + v1 * I1 + 0.5 * g1 * I1 ** 2 + g2 * I2 + 2.0 * (v2 + g2 * I1) * c33 + 4.0 * g3 * c33 ** 2
            dce = 2.0 * (v2 + g2 * I1) + 4.0 * g4 * c33
            ds33 = dcI + dce * c33 + ce + 4.0 * g3 * c33 ** 2 + 2.0 * ce2 * c33
            if cap is not None:
                s33 = s33 + 2.0 * Gt * (e33 - c33) * w
                ds33 = ds33 + 2.0 * Gt * w
            delta = -s33 / (ds33 + 1e-12)
            if not np.all(np.isfinite(delta)):
                raise FloatingPointError("landau_stress_2d: non-finite e33 Newton update")
            e33 = e33 + delta
            if np.all(np.abs(delta) < 1e-9):
                break
        if e33_state is not None:
            e33_state["e33"] = e33
    else:
        e33 = np.zeros_like(a11)
        I1, I2, c11, c22, c12, c21, c33, w, cI, ce, ce2 = _landau_scalars_2d(a11, a22, a12, a21, e33, lam, mu, v, cap)
    cross = c12 * c21
    t_ip = c11 + c22
    sig = np.empty(e.shape)
    sig[..., 0, 0] = cI + ce * c11 + ce2 * (c11 * c11 + cross)
    sig[..., 1, 1] = cI + ce * c22 + ce2 * (c22 * c22 + cross)
    sig[..., 0, 1] = ce * c12 + ce2 * (c12 * t_ip)
    sig[..., 1, 0] = ce * c21 + ce2 * (c21 * t_ip)
    if cap is not None:
        r = 2.0 * Gt * w
        sig[..., 0, 0] += r * (a11 - c11)
        sig[..., 1, 1] += r * (a22 - c22)
        sig[..., 0, 1] += r * (a12 - c12)
        sig[..., 1, 0] += r * (a21 - c21)
    return sig


def landau_stress_2d_root(e, lam, mu, v, cap_type=None, cap_limit=None, cap_ratio=0.1, cap_power=1.0):
    """The plane-stress Landau stress at the root of sigma33 = 0: the
    reference's Newton steps (landau_stress_2d) repeated from the stepped e33
    until no voxel's e33 moves by 1e-15, from the linear guess; the stress of
    the last evaluation.  The reference reaches this state only over its
    solver's iterations (its e33 lags by its last step); the GPU kernels
    solve for it at every evaluation."""
    a11, a22 = e[..., 0, 0], e[..., 1, 1]
    e33 = -lam / (lam + 2.0 * mu) * (a11 + a22)
    sig = None
    for _ in range(200):
        st = {"e33": e33}
        sig = landau_stress_2d(e, lam, mu, v, cap_type, cap_limit, cap_ratio, cap_power, True, st)
        moved = np.max(np.abs(st["e33"] - e33))
        e33 = st["e33"]
        if moved < 1e-15:
            break
    return sig


def anderson_step(hist_g, hist_f, g, f, m):
    """Type-II Anderson mixing of the last m + 1 fixed-point images and
    residuals (mgkmc/linear_elastic_simulator.py:1185-1209): returns the next
    iterate and the trimmed history; a non-finite mix gives the plain step
    and restarts the history from the last pair."""
    hist_g.append(g.reshape(-1))
    hist_f.append(f.reshape(-1))
    if len(hist_f) > m + 1:
        hist_g.pop(0)
        hist_f.pop(0)
    if len(hist_f) < 2:
        return g, hist_g, hist_f
    dF = np.stack([hist_f[i + 1] - hist_f[i] for i in range(len(hist_f) - 1)], axis=1)
    dG = np.stack([hist_g[i + 1] - hist_g[i] for i in range(len(hist_g) - 1)], axis=1)
    try:
        gam = np.linalg.lstsq(dF, hist_f[-1], rcond=None)[0]
        x = hist_g[-1] - dG @ gam
    except np.linalg.LinAlgError:
        x = None
    if x is not None and np.all(np.isfinite(x)):
        return x.reshape(g.shape), hist_g, hist_f
    return g, hist_g[-1:], hist_f[-1:]


def spectral_solver_landau_2d(lam, mu, v, eps_bar, eps_plastic=None, max_iter=400, tol=1e-6, pixel=1.0,
                              eps_init=None, anderson_m=5, cap_type=None, cap_limit=None, cap_ratio=0.1,
                              cap_power=1.0, return_info=False, plane_stress=False, e33_state=None,
                              e33_root=False):
    """Landau small-strain LS fixed point (plane strain, or plane stress with
    the e33 Newton solve and its warm state e33_state; e33_root: e33 solved
    to its root at every evaluation instead), the basic scheme
    with Anderson mixing (mgkmc/linear_elastic_simulator.py:952-1228, solver
    "dbfft"): medium (mean lam, mean mu) fixed; G(eps) = eps_bar + Gamma0 *
    (sigma_L(eps - eps_p) - C0:eps) with zero-mean fluctuation; stop when
    |G(eps) - eps| / |eps| < tol (eps = G(eps)); otherwise mix the history.
    A non-finite update raises FloatingPointError."""
    lam0, mu0 = float(np.mean(lam)), float(np.mean(mu))
    shape = np.shape(lam)
    axes = (0, 1)
    G = green_operator(wave_vectors(shape, pixel), lam0, mu0)
    if eps_init is not None:
        eps = eps_init.copy()
        eps += eps_bar - eps_init.mean(axis=axes)
    else:
        eps = np.broadcast_to(eps_bar, shape + (2, 2)).copy()
    ep = eps_plastic
    if plane_stress and e33_root:  # e33 at the root at every evaluation
        law = lambda x: landau_stress_2d_root(x - ep if ep is not None else x, lam, mu, v, cap_type, cap_limit,
                                              cap_ratio, cap_power)
    else:
        law = lambda x: landau_stress_2d(x - ep if ep is not None else x, lam, mu, v, cap_type, cap_limit, cap_ratio,
                                         cap_power, plane_stress, e33_state)
    hg, hf = [], []
    it_done, diff = 0, np.inf
    for it in range(max_iter):
        tau = law(eps) - hooke(eps, lam0, mu0, 2)
        tau_hat = np.fft.fftn(tau, axes=axes, norm="ortho")
        et = np.fft.ifftn(-np.einsum("xykhij,xyij->xykh", G, tau_hat), axes=axes, norm="ortho").real
        et -= et.mean(axis=axes)
        eps_new = eps_bar + et
        diff = np.linalg.norm(eps_new - eps) / (np.linalg.norm(eps) + 1e-20)
        it_done = it + 1
        if not np.isfinite(diff):
            raise FloatingPointError("spectral_solver_landau_2d: non-finite strain update in LS loop")
        if diff < tol:
            eps = eps_new
            break
        if anderson_m > 0:
            eps, hg, hf = anderson_step(hg, hf, eps_new, eps_new - eps, anderson_m)
        else:
            eps = eps_new
    sig_out = law(eps)
    out = (eps, sig_out, eps.mean(axis=axes), sig_out.mean(axis=axes))
    return out + (it_done, diff) if return_info else out


def landau_stress_3d(e, lam, mu, v, cap_type=None, cap_limit=None, cap_ratio=0.1, cap_power=1.0):
    """Landau small-strain stress in 3D (mgkmc/elasticity.py:811-857) with the
    strain capping of :297-334: sigma = cI I + ce e + ce2 e^2 from the
    invariants I1 = tr e, I2 = tr e^2, I3 = tr e^3 of the (capped) strain,
    cI = lam I1 + v1/2 I1^2 + v2 I2 + g1/6 I1^3 + g2 I1 I2 + 4/3 g3 I3,
    ce = 2 (mu + v2 I1 + g2/2 I1^2 + g4 I2), ce2 = 4 (v3 + g3 I1); capping as
    in landau_stress_2d with the 3D deviator."""
    v1, v2, v3, g1, g2, g3, g4 = v
    eye = np.eye(3)
    w = None
    if cap_type is not None:
        I1a = np.trace(e, axis1=-2, axis2=-1)
        dev = e - (1.0 / 3.0) * I1a[..., None, None] * eye
        E_eq = np.sqrt(np.maximum(0.0, (2.0 / 3.0) * np.einsum("...ij,...ji->...", dev, dev)))
        mu_mean = np.mean(mu)
        E_cap = cap_limit if cap_limit is not None and cap_limit > 0 else (
            np.sqrt(0.2 * mu_mean / abs(g4)) if g4 < 0 else 999.0)
        f = np.ones_like(E_eq)
        nz = E_eq > 1e-12
        if cap_type == "smooth":
            rp = np.minimum(100.0, (E_eq[nz] / E_cap) ** cap_power)
            f[nz] = (E_cap / E_eq[nz]) * np.tanh(rp) ** (1.0 / cap_power)
            w = np.tanh(np.minimum(100.0, (E_eq / E_cap) ** cap_power)) ** 2
        else:
            capped = E_eq > E_cap
            np.divide(E_cap, E_eq, out=f, where=capped)
            w = capped.astype(float)
        c = dev * f[..., None, None] + (1.0 / 3.0) * I1a[..., None, None] * eye
    else:
        c = e
    I1 = np.trace(c, axis1=-2, axis2=-1)
    c2 = np.einsum("...ij,...jk->...ik", c, c)
    I2 = np.trace(c2, axis1=-2, axis2=-1)
    I3 = np.trace(np.einsum("...ij,...jk->...ik", c2, c), axis1=-2, axis2=-1)
    cI = lam * I1 + 0.5 * v1 * I1 ** 2 + v2 * I2 + (1.0 / 6.0) * g1 * I1 ** 3 + g2 * I1 * I2 + (4.0 / 3.0) * g3 * I3
    ce = 2.0 * (mu + v2 * I1 + 0.5 * g2 * I1 ** 2 + g4 * I2)
    ce2 = 4.0 * (v3 + g3 * I1)
    sig = cI[..., None, None] * eye + ce[..., None, None] * c + ce2[..., None, None] * c2
    if cap_type is not None:
        sig += 2.0 * (cap_ratio * np.asarray(mu))[..., None, None] * (e - c) * w[..., None, None]
    return sig


def spectral_solver_landau_3d(lam, mu, v, eps_bar, eps_plastic=None, max_iter=400, tol=1e-6, pixel=1.0,
                              eps_init=None, cap_type=None, cap_limit=None, cap_ratio=0.1, cap_power=1.0,
                              return_info=False):
    """3D Landau small-strain LS fixed point (mgkmc/linear_elastic_simulator.py:
    1231-1350): medium (mean lam, mean mu); eps <- eps_bar + zero-mean
    Gamma0 * (sigma_L(eps - eps_p) - C0:eps); stop when the relative update
    is below tol (the basic scheme, no mixing)."""
    lam0, mu0 = float(np.mean(lam)), float(np.mean(mu))
    shape = np.shape(lam)
    axes = (0, 1, 2)
    G = green_operator(wave_vectors(shape, pixel), lam0, mu0)
    if eps_init is not None:
        eps = eps_init.copy()
        eps += eps_bar - eps_init.mean(axis=axes)
    else:
        eps = np.broadcast_to(eps_bar, shape + (3, 3)).copy()
    ep = eps_plastic
    law = lambda x: landau_stress_3d(x - ep if ep is not None else x, lam, mu, v, cap_type, cap_limit, cap_ratio,
                                     cap_power)
    it_done, diff = 0, np.inf
    for it in range(max_iter):
        tau = law(eps) - hooke(eps, lam0, mu0, 3)
        tau_hat = np.fft.fftn(tau, axes=axes, norm="ortho")
        et = np.fft.ifftn(-np.einsum("xyzkhij,xyzij->xyzkh", G, tau_hat), axes=axes, norm="ortho").real
        et -= et.mean(axis=axes)
        eps_new = eps_bar + et
        diff = np.linalg.norm(eps_new - eps) / (np.linalg.norm(eps) + 1e-20)
        eps = eps_new
        it_done = it + 1
        if not np.isfinite(diff):
            raise FloatingPointError("spectral_solver_landau_3d: non-finite strain update in LS loop")
        if diff < tol:
            break
    sig_out = law(eps)
    out = (eps, sig_out, eps.mean(axis=axes), sig_out.mean(axis=axes))
    return out + (it_done, diff) if return_info else out


def rose_stress_2d(e, lam, mu, eta, floor_f=0.1, plane_mode="plane_strain"):
    """Rose secant-modulus stress (mgkmc/elasticity.py:868-944): G = max(mu
    exp(-eta eq), floor mu), K = lam + 2 mu / 3 kept; plane stress: eps_zz by
    five fixed-point steps; sigma_yx copied from sigma_xy."""
    exx, eyy, exy = e[..., 0, 0], e[..., 1, 1], e[..., 0, 1]
    K = lam + (2.0 / 3.0) * mu

    def eq_of(ezz):
        tr3 = (exx + eyy + ezz) / 3.0
        return np.sqrt((2.0 / 3.0) * ((exx - tr3) ** 2 + (eyy - tr3) ** 2 + (ezz - tr3) ** 2 + 2.0 * exy ** 2))

    def g_of(eq):
        return np.maximum(mu * np.exp(-eta * eq), floor_f * mu)

    ezz = np.zeros_like(exx)
    if plane_mode == "plane_stress":
        ezz = -lam / (lam + 2.0 * mu) * (exx + eyy)
        for _ in range(5):
            g = g_of(eq_of(ezz))
            ezz = -((3.0 * K - 2.0 * g) / (3.0 * K + 4.0 * g)) * (exx + eyy)
    G = g_of(eq_of(ezz))
    tr = exx + eyy + ezz
    le = K - (2.0 / 3.0) * G
    sig = np.zeros_like(e)
    sig[..., 0, 0] = le * tr + 2.0 * G * exx
    sig[..., 1, 1] = le * tr + 2.0 * G * eyy
    sig[..., 0, 1] = 2.0 * G * exy
    sig[..., 1, 0] = sig[..., 0, 1]
    return sig


def spectral_solver_rose_2d(lam, mu, eta, floor_f, eps_bar, eps_plastic=None, max_iter=400, tol=1e-6, pixel=1.0,
                            plane_mode="plane_strain", eps_init=None, return_info=False):
    """Rose-law LS fixed point (mgkmc/linear_elastic_simulator.py:852-950):
    reference medium (mean lam, (mean mu + floor mean mu) / 2)."""
    lam0 = float(np.mean(lam))
    mu_avg = float(np.mean(mu))
    mu0 = 0.5 * (mu_avg + floor_f * mu_avg)
    shape = np.shape(lam)
    axes = (0, 1)
    G = green_operator(wave_vectors(shape, pixel), lam0, mu0)
    if eps_init is not None:
        eps = eps_init.copy()
        eps += eps_bar - eps_init.mean(axis=axes)
    else:
        eps = np.broadcast_to(eps_bar, shape + (2, 2)).copy()
    ep = eps_plastic
    it_done, diff = 0, np.inf
    for it in range(max_iter):
        sig = rose_stress_2d(eps - ep if ep is not None else eps, lam, mu, eta, floor_f, plane_mode)
        tau = sig - hooke(eps, lam0, mu0, 2)
        tau_hat = np.fft.fftn(tau, axes=axes, norm="ortho")
        et = np.fft.ifftn(-np.einsum("xykhij,xyij->xykh", G, tau_hat), axes=axes, norm="ortho").real
        et -= et.mean(axis=axes)
        eps_new = eps_bar + et
        diff = np.linalg.norm(eps_new - eps) / (np.linalg.norm(eps) + 1e-20)
        eps = eps_new
        it_done = it + 1
        if diff < tol:
            break
    sig_out = rose_stress_2d(eps - ep if ep is not None else eps, lam, mu, eta, floor_f, plane_mode)
    out = (eps, sig_out, eps.mean(axis=axes), sig_out.mean(axis=axes))
    return out + (it_done, diff) if return_info else out


def equilibrium_residual(eps, E, nu, eps_bar, eps_plastic=None, pixel=1.0, plane_mode="plane_strain"):
    """|| eps_bar - Gamma0 * tau(eps) - eps || / ||eps||: the fixed-point defect
    of the LS equation, which is zero exactly at mechanical equilibrium."""
    d = E.ndim
    axes = tuple(range(d))
    E_avg, nu_avg = E.mean(), nu.mean()
    if d == 2:
        lam, mu = lame_2d(E, nu, plane_mode)
        lam0, mu0 = lame_2d(E_avg, nu_avg, plane_mode)
    else:
        lam, mu = lame_3d(E, nu)
        lam0, mu0 = lame_3d(E_avg, nu_avg)
    G = green_operator(wave_vectors(E.shape, pixel), lam0, mu0)
    sub = "xyz"[:d]
    ep = eps_plastic
    tau = hooke(eps - ep if ep is not None else eps, lam, mu, d) - hooke(eps, lam0, mu0, d)
    et = np.fft.ifftn(-np.einsum(f"{sub}khij,{sub}ij->{sub}kh", G,
                                 np.fft.fftn(tau, axes=axes, norm="ortho")),
                      axes=axes, norm="ortho").real
    et -= et.mean(axis=axes)
    return np.linalg.norm(eps_bar + et - eps) / (np.linalg.norm(eps) + 1e-20)


def mixed_bc_solve_2d(E, nu, eps_plastic, strain_mask, target, tol_ls=1e-10, max_iter_ls=500,
                      tol_macro=1e-4, max_iter_macro=20, pixel=1.0, plane_mode="plane_strain",
                      eps_bar0=None, eps_warm=None):
    """Mixed stress/strain macro loop (linear_elastic_simulator.py:176-197,
    :150-152) around the warm-started LS solve, with an eigenstrain field.

    strain_mask (2,2) bool: True where eps_bar is prescribed; elsewhere the mean
    stress is driven to ``target``.  ``eps_bar0``/``eps_warm`` carry the macro
    strain and the warm-start field of a previous load step (:170, :199).  Returns (eps, sig, eps_bar, sig_mean,
    macro_iters, total_ls_iters)."""
    E_avg, nu_avg = E.mean(), nu.mean()
    stress_mask = ~strain_mask
    eps_bar = np.zeros((2, 2)) if eps_bar0 is None else np.array(eps_bar0, dtype=np.float64)
    total = 0
    for it_macro in range(max_iter_macro):
        eps_bar[strain_mask] = target[strain_mask]
        eps, sig, epsM, sigM, its, _ = spectral_solver(
            E, nu, eps_bar, eps_plastic, max_iter=max_iter_ls, tol=tol_ls, pixel=pixel,
            plane_mode=plane_mode, eps_init=eps_warm, return_info=True)
        total += its
        eps_warm = eps
        err = np.zeros((2, 2))
        err[stress_mask] = target[stress_mask] - sigM[stress_mask]
        max_err = np.max(np.abs(err[stress_mask])) if np.any(stress_mask) else 0.0
        if max_err < tol_macro:
            return eps, sig, eps_bar.copy(), sigM, it_macro + 1, total
        d_eps = (err - nu_avg * np.trace(err) * np.eye(2)) / E_avg
        eps_bar[stress_mask] += d_eps[stress_mask]
    return eps, sig, eps_bar.copy(), sigM, max_iter_macro, total
