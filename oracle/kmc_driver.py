"""numpy restatement of the 2D KMC/AQS trajectory (oracle).

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).

Follows KmcSimulation2D.run_simulation (mgkmc/kmc_simulator.py:796-1157) on
the path the benchmark exercises: small-strain linear elasticity, KMC mode
(cascade off, or on: ``cascade_mode``), no thermal conduction, fast
patching off or on (``fast_patching``), redraw of both directions and
barriers after a flip.  Fast patching (:229-261, :1044-1074, :764-792,
:1094-1096) replaces the LS re-solve after a flip by a local stress patch
and a uniform shift, with a full re-solve every ``sync_interval`` KMC flips
and after each cascade.  Cascade mode
(:876-889, _run_cascade :577-794, linear small-strain branch :728-784):
after each barrier update, while modes with Q < stability_threshold exist,
flip in one batch the most unstable mode of each voxel that has one (modes
sorted by Q ascending, first per voxel), each with the flip bookkeeping and
redraws of a KMC event, then one LS re-solve; rates then use only modes with
q > 0 (compute_rates_2d cascade_mode=True).  Per event: update_barriers (:874 ->
compute_barrier_2d), compute_rates_2d (:891), the waiting time (:893), the
clock/strain advance (:895-898), selection + decode (:899-900), the flip and
its bookkeeping (:1025-1042), and a cold-started LS re-solve (:1076, which
passes no warm start).  After each AQS step, the mixed stress-control loop
(:1106-1143).  The NaN / |sigma| > 20 GPa guard of elastic_run (:522-524)
raises ValueError.

Draws come from an explicit numpy Generator in a fixed order instead of the
reference's two global streams (numpy for t_wait and redraws, numba's for
selection): per attempt u_wait; per event u_sel, then M orientations
theta ~ U[0, pi) and M barriers N(q_mean, q_std) clipped below at q_min; per
cascade flip (in batch order) the same M + M redraws.  The GPU driver
consumes the same draws in the same order.
"""
import numpy as np

from . import kmc as OK
from . import ls as OL


def pure_shear_modes(theta, gamma0):
    c, s = np.cos(2 * theta), np.sin(2 * theta)
    cat = np.empty(theta.shape + (2, 2))
    cat[..., 0, 0] = 0.5 * gamma0 * c
    cat[..., 1, 1] = -0.5 * gamma0 * c
    cat[..., 0, 1] = 0.5 * gamma0 * s
    cat[..., 1, 0] = 0.5 * gamma0 * s
    return cat


class GeneratorDraws:
    """The driver's draws from an explicit numpy Generator, in a fixed order:
    per attempt u_wait; per event u_sel, then M orientations theta ~ U[0, pi)
    (pure-shear modes of amplitude gamma0/2) and M barriers N(q_mean, q_std)
    clipped below at q_min."""

    def __init__(self, rng, gamma0, q_mean, q_std, q_min):
        self.rng, self.gamma0, self.q = rng, gamma0, (q_mean, q_std, q_min)

    def u_wait(self):
        return self.rng.random()

    def u_sel(self):
        return self.rng.random()

    def catalog(self, M):
        return pure_shear_modes(self.rng.uniform(0.0, np.pi, M), self.gamma0)

    def q0(self, M):
        return np.clip(self.rng.normal(self.q[0], self.q[1], M), self.q[2], None)


class ReferenceDraws:
    """The reference's own draws, taken from a numpy RandomState standing for
    its global stream, call for call: t_wait = -ln(rand()) / total
    (kmc_simulator.py:893); the selection threshold uniform(0, total)
    (kmc_simulator_functions.py:62, = total * U, which the selection takes as
    u = U); the redrawn catalog stz_catalog_glass_2d (:78-98: per mode
    gxx = 0.5 gamma0 N(0,1), then gxy = 0.5 gamma0 N(0,1), pure shear); the
    redrawn barriers of the Gaussian generator (:222-229: normal(mean, std,
    size=M) clipped to [min_cutoff, max_cutoff])."""

    def __init__(self, rs, gamma0, mean, std, min_cutoff=None, max_cutoff=None):
        self.rs, self.gamma0 = rs, gamma0
        self.mean, self.std, self.lo, self.hi = mean, std, min_cutoff, max_cutoff

    def u_wait(self):
        return self.rs.rand()

    def u_sel(self):
        return self.rs.uniform(0.0, 1.0)

    def catalog(self, M):
        cat = np.zeros((M, 2, 2))
        for i in range(M):
            gxx = 0.5 * self.gamma0 * self.rs.normal()
            gxy = 0.5 * self.gamma0 * self.rs.normal()
            cat[i, 0, 0], cat[i, 1, 1] = gxx, -gxx
            cat[i, 0, 1] = cat[i, 1, 0] = gxy
        return cat

    def q0(self, M):
        b = self.rs.normal(loc=self.mean, scale=self.std, size=(M,))
        if self.lo is not None or self.hi is not None:
            b = np.clip(b, self.lo, self.hi)
        return b


def patch_kernels_2d(E, nu, R, max_iter=200, tol=1e-6, pixel=1.0, plane_mode="plane_strain"):
    """Stress patches of the fast-patching mode (kmc_simulator.py:229-261).

    For each deviatoric basis P0 = [[1, 0], [0, -1]] and P1 = [[0, 1], [1, 0]]:
    the LS stress response to a unit eigenstrain P at the voxel
    (nx//2, ny//2) under zero macro strain, read in the (2R+1)^2 window centred
    on that voxel (periodic), and the part of its mean that the window
    misses: mean(sigma) - sum(window) / (nx*ny).  Returns
    (kernels (2, 2R+1, 2R+1, 2, 2), missing_mean (2, 2, 2))."""
    nx, ny = E.shape
    bases = (np.array([[1.0, 0.0], [0.0, -1.0]]), np.array([[0.0, 1.0], [1.0, 0.0]]))
    ix = (np.arange(-R, R + 1) + nx // 2) % nx
    iy = (np.arange(-R, R + 1) + ny // 2) % ny
    kernels = np.zeros((2, 2 * R + 1, 2 * R + 1, 2, 2))
    missing = np.zeros((2, 2, 2))
    for b, P in enumerate(bases):
        ep = np.zeros((nx, ny, 2, 2))
        ep[nx // 2, ny // 2] = P
        _, sig, _, _ = OL.spectral_solver(E, nu, np.zeros((2, 2)), ep, max_iter=max_iter, tol=tol,
                                          pixel=pixel, plane_mode=plane_mode)
        kernels[b] = sig[ix[:, None], iy[None, :]]
        missing[b] = np.mean(sig, axis=(0, 1)) - np.sum(kernels[b], axis=(0, 1)) / (nx * ny)
    return kernels, missing


def apply_patch_2d(sig, x, y, gxx, gxy, kernels, missing, unit=None, scale=0.0):
    """One fast-patching stress update in place (kmc_simulator.py:1052-1069,
    cascade branch :764-774): sig += unit * scale (when ``unit`` is given), then
    the window gxx*K0 + gxy*K1 added around (x, y) with periodic wrap in (dx, dy)
    order, then the missing mean gxx*m0 + gxy*m1 added everywhere."""
    nx, ny = sig.shape[:2]
    R = (kernels.shape[1] - 1) // 2
    if unit is not None:
        sig += unit * scale
    patch = gxx * kernels[0] + gxy * kernels[1]
    shift = gxx * missing[0] + gxy * missing[1]
    px = (x + np.arange(-R, R + 1)) % nx
    py = (y + np.arange(-R, R + 1)) % ny
    # unbuffered adds in (dx, dy) order: repeated voxels (window wider than the
    # grid) accumulate in the reference's loop order
    np.add.at(sig, (px[:, None], py[None, :]), patch)
    sig += shift


def run_kmc2d(E, nu, catalog, Q0, rng, n_steps, max_events=None, gamma0=0.1, T=300.0, nu0=1e13,
              strain_rate=1e7, step_size=1e-5, q_act_temp=0.37, jp=0.0, jt=0.0, cap=2.0, jn=0.0,
              stress_targets=None, mixed_tol=1e4, mixed_max_iter=50, ls_tol=1e-6, ls_max_iter=200,
              q_mean=1.0, q_std=0.15, q_min=0.3, volume=1.0, cascade_mode=False, stability_threshold=0.0,
              max_cascade_steps_pct=0.3, fast_patching=None, eps_macro0=None):
    """``rng``: a numpy Generator (``GeneratorDraws``) or a draws object
    (``ReferenceDraws``).  ``eps_macro0``: the simulator's macro strain when
    the run starts (the reference's run_simulation starts from
    ``self.eps_macro``, :869, zero for a fresh simulator)."""
    nx, ny, M = Q0.shape
    draws = rng if hasattr(rng, "u_wait") else GeneratorDraws(rng, gamma0, q_mean, q_std, q_min)
    stress_targets = {(1, 1): 0.0} if stress_targets is None else stress_targets
    catalog = catalog.copy()
    Q0 = Q0.copy()
    eps_p = np.zeros((nx, ny, 2, 2))
    soft = np.zeros((nx, ny, 2))
    t_last = np.full((nx, ny), -np.inf)
    prev = np.zeros((nx, ny, 2, 2))
    Q = np.zeros((nx, ny, M))
    eps_macro = np.zeros((2, 2)) if eps_macro0 is None else np.array(eps_macro0, dtype=np.float64).reshape(2, 2)
    time = 0.0
    tau = 1.0 / (nu0 * np.exp(-q_act_temp / (OK.KB * T))) if T > 0 else np.inf  # kmc_simulator.py:86-92
    E_avg, nu_avg = E.mean(), nu.mean()

    def elastic_run():
        eps, sig, _, sigM = OL.spectral_solver(E, nu, eps_macro, eps_p, max_iter=ls_max_iter, tol=ls_tol)
        if np.any(np.isnan(sig)) or np.max(np.abs(sigM)) / 1e9 > 20.0:
            raise ValueError(f"Unstable stress in small-strain elastic_run: {sigM / 1e9} GPa")
        return sig, sigM

    # fast patching (kmc_simulator.py:76-80, :170-171): patches computed once
    # from the initial moduli; the unit macro-strain response is computed at
    # the first KMC flip (:1045-1050)
    fast = bool(fast_patching and fast_patching.get("enabled", False))
    if fast:
        R = int(fast_patching.get("patch_radius", 5))
        sync_interval = int(fast_patching.get("sync_interval", 100))
        kernels, missing = patch_kernels_2d(E, nu, R, max_iter=ls_max_iter, tol=ls_tol)
    sig_unit = None
    flips_since_sync = 0

    sig, sigM = elastic_run()
    events = []
    cascade_flips = []  # (x, y, m, time, batch)
    n_solves = 1
    max_cascade_limit = int(max_cascade_steps_pct * nx * ny)  # kmc_simulator.py:815
    cascade_count = 0
    n_batches = 0

    def result():
        return dict(events=events, eps_macro=eps_macro, sig=sig, eps_p=eps_p, time=time, steps=steps_done,
                    solves=n_solves, catalog=catalog, Q0=Q0, cascade_flips=cascade_flips)

    def flip(x, y, m):
        C = catalog[x, y, m].copy()
        OK.apply_flip_2d(eps_p, soft, t_last, catalog, x, y, m, time, jp, jt, cap, jn)
        prev[x, y] = C
        catalog[x, y] = draws.catalog(M)
        Q0[x, y] = draws.q0(M)
    strain_unit = np.zeros((2, 2))
    strain_unit[0, 0] = 1.0
    dt_step = abs(step_size) / strain_rate if strain_rate > 0 else 1.0
    remaining = 0.0
    steps_done = 0
    while steps_done < n_steps:
        remaining += dt_step
        while remaining > 0:
            OK.compute_barrier(Q, Q0, sig, catalog, volume, soft, t_last, time, prev, cap, 0, tau)
            if cascade_mode and np.any(Q < stability_threshold):
                # _run_cascade: batches until no mode is unstable
                local_step, flips = 0, 0
                while True:
                    OK.compute_barrier(Q, Q0, sig, catalog, volume, soft, t_last, time, prev, cap, 0, tau)
                    uns = OK.find_unstable_2d(Q, stability_threshold)  # (x, y, m) order
                    if len(uns) == 0:
                        break
                    flat = (uns[:, 0] * ny + uns[:, 1]) * M + uns[:, 2]
                    order = flat[np.argsort(Q.reshape(-1)[flat])]
                    seen, batch = set(), []
                    for f in order:
                        v = int(f) // M
                        if v not in seen:
                            seen.add(v)
                            batch.append(OK.decode_index_2d(int(f), ny, M))
                    for (x, y, m) in batch:
                        flip(x, y, m)
                        cascade_flips.append((x, y, m, time, n_batches))
                        if fast:
                            # the patch uses the redrawn mode (:764-774)
                            apply_patch_2d(sig, x, y, catalog[x, y, m, 0, 0], catalog[x, y, m, 0, 1],
                                           kernels, missing)
                    if not fast:
                        sig, sigM = elastic_run()
                        n_solves += 1
                    n_batches += 1
                    flips += len(batch)
                    local_step += 1
                    if local_step > nx * ny:
                        break
                if fast and flips > 0:
                    # corrector: the final sync (:790-792)
                    sig, sigM = elastic_run()
                    n_solves += 1
                if flips > 0:
                    cascade_count += 1
                if cascade_count > max_cascade_limit:
                    return result()
                continue
            cascade_count = 0
            rates, indices, total = OK.compute_rates(Q, 1.0, T, nu0, cascade_mode=cascade_mode)
            if total > 0:
                u = draws.u_wait()
                t_wait = -np.log(u) / total
                if t_wait < remaining:
                    time += t_wait
                    eps_macro += strain_unit * (strain_rate * t_wait)
                    remaining -= t_wait
                    k = OK.select_event(rates, total, draws.u_sel())
                    x, y, m = OK.decode_index_2d(int(indices[k]), ny, M)
                    C = catalog[x, y, m].copy()
                    flip(x, y, m)
                    if fast:
                        if sig_unit is None:
                            _, sig_unit, _, _ = OL.spectral_solver(E, nu, strain_unit, np.zeros_like(eps_p),
                                                                   max_iter=ls_max_iter, tol=ls_tol)
                        apply_patch_2d(sig, x, y, C[0, 0], C[0, 1], kernels, missing,
                                       unit=sig_unit if t_wait > 0 else None, scale=strain_rate * t_wait)
                        flips_since_sync += 1
                        if flips_since_sync >= sync_interval:
                            sig, sigM = elastic_run()
                            n_solves += 1
                            flips_since_sync = 0
                    else:
                        sig, sigM = elastic_run()
                        n_solves += 1
                    events.append((x, y, m, time))
                    if max_events is not None and len(events) >= max_events:
                        return result()
                    continue
            if fast and sig_unit is not None:
                sig += sig_unit * (strain_rate * remaining)
            eps_macro += strain_unit * (strain_rate * remaining)
            time += remaining
            remaining = 0.0
        # mixed stress control at the end of the AQS step (kmc_simulator.py:1106-1143)
        prev_e, prev_s = {}, {}
        for _ in range(mixed_max_iter):
            sig, sigM = elastic_run()
            n_solves += 1
            err = np.zeros((2, 2))
            err_max = 0.0
            for idx, target in stress_targets.items():
                e = target - sigM[idx]
                err[idx] = e
                err_max = max(err_max, abs(e))
            if err_max < mixed_tol:
                break
            d_eps = (err - nu_avg * np.trace(err) * np.eye(2)) / E_avg
            for idx in stress_targets:
                step = d_eps[idx]
                if idx in prev_e:
                    d_e = eps_macro[idx] - prev_e[idx]
                    d_s = sigM[idx] - prev_s[idx]
                    if abs(d_e) > 1e-14 and np.isfinite(d_s):
                        slope = d_s / d_e
                        if np.isfinite(slope) and slope > 0.01 * E_avg:
                            step = err[idx] / slope
                prev_e[idx] = eps_macro[idx]
                prev_s[idx] = sigM[idx]
                eps_macro[idx] += step
        steps_done += 1
    return result()


# ----------------------------------------------------------------- 3D ---
def in_plane_modes(theta, gamma0):
    """(M, 3, 3) in-plane pure-shear modes (the glass mode of
    stz/catalog.py:7-29 with a fixed amplitude gamma0/2 and orientation theta)."""
    c, s = np.cos(2 * theta), np.sin(2 * theta)
    cat = np.zeros(theta.shape + (3, 3))
    cat[..., 0, 0] = 0.5 * gamma0 * c
    cat[..., 1, 1] = -0.5 * gamma0 * c
    cat[..., 0, 1] = 0.5 * gamma0 * s
    cat[..., 1, 0] = 0.5 * gamma0 * s
    return cat


class GeneratorDraws3D(GeneratorDraws):
    """GeneratorDraws with (M, 3, 3) in-plane modes."""

    def catalog(self, M):
        return in_plane_modes(self.rng.uniform(0.0, np.pi, M), self.gamma0)


class ReferenceDraws3D(ReferenceDraws):
    """The 3D simulator's draws (aqs.py): t_wait from uniform() (:880), the
    selection's uniform(0, total) (stz/kmc.py:84), the catalog of
    stz_catalog_glass (stz/catalog.py:7-40: per mode gxx = 0.5 gamma0 N(0,1),
    then gxy, in-plane pure shear), Gaussian barriers
    (stz/barrier_generators.py:24-29)."""

    def u_wait(self):
        return self.rs.uniform()

    def catalog(self, M):
        cat = np.zeros((M, 3, 3))
        cat[:, :2, :2] = super().catalog(M)
        return cat


def run_kmc3d(E, nu, catalog, Q0, rng, n_steps, max_events=None, gamma0=0.1, T=300.0, nu0=1e13, strain_rate=1e7,
              step_size=1e-5, q_act_temp=0.37, jp=0.0, jt=0.0, cap=2.0, jn=0.0, component=(0, 0),
              stress_targets=None, mixed_tol=1e4, mixed_max_iter=50, ls_tol=1e-6, ls_max_iter=200, q_mean=1.0,
              q_std=0.15, q_min=0.3, volume=1.0, eps_macro0=None):
    """ThermalSimulation.run_simulation (aqs.py:682-1201) on the small-strain
    KMC path (no cascade, no fast patching, no conduction; redraw of the
    voxel's catalog and barriers after a flip): per attempt update_barriers
    (:455-460), compute_rates (:873), the waiting time (:877-881), selection
    and decode (:889-892), apply_flip_soa and prev_strain_dir (:996-997), the
    redraws (:1006-1013) and update_stresses (:1073, the LS re-solve of
    update_stress_fft_full :349); at the end of an AQS step update_stresses
    (:1097) and the mixed loop (:1118-1152): the full correction
    (sigma_err - nu_avg tr I) / E_avg with the driven component zeroed, added
    to eps_macro, then a re-solve.  Default stress targets for driving
    component (0, 0): yy and zz stress-free (:715-722)."""
    nx, ny, nz, M = Q0.shape
    draws = rng if hasattr(rng, "u_wait") else GeneratorDraws3D(rng, gamma0, q_mean, q_std, q_min)
    if stress_targets is None:
        stress_targets = {(1, 1): 0.0, (2, 2): 0.0} if tuple(component) == (0, 0) else \
            {(0, 0): 0.0, (1, 1): 0.0, (2, 2): 0.0}
    catalog, Q0 = catalog.copy(), Q0.copy()
    eps_p = np.zeros((nx, ny, nz, 3, 3))
    soft = np.zeros((nx, ny, nz, 4))
    t_last = np.full((nx, ny, nz), -np.inf)
    prev = np.zeros((nx, ny, nz, 3, 3))
    Q = np.zeros((nx, ny, nz, M))
    eps_macro = np.zeros((3, 3)) if eps_macro0 is None else np.array(eps_macro0, dtype=np.float64).reshape(3, 3)
    time = 0.0
    tau = 1.0 / (nu0 * np.exp(-q_act_temp / (OK.KB * T))) if T > 0 else np.inf
    E_avg, nu_avg = np.mean(E), np.mean(nu)
    unit = np.zeros((3, 3))
    unit[tuple(component)] = 1.0
    n_solves = 0

    def update_stresses():
        nonlocal n_solves
        n_solves += 1
        _, s, _, _ = OL.spectral_solver(E, nu, eps_macro, eps_p, max_iter=ls_max_iter, tol=ls_tol)
        return s

    sig = update_stresses()
    events = []
    dt_step = abs(step_size) / strain_rate if strain_rate > 0 else 1.0
    remaining = 0.0
    steps_done = 0

    def result():
        return dict(events=events, eps_macro=eps_macro, sig=sig, eps_p=eps_p, time=time, steps=steps_done,
                    solves=n_solves, catalog=catalog, Q0=Q0)

    while steps_done < n_steps:
        remaining += dt_step
        while remaining > 0:
            OK.compute_barrier(Q, Q0, sig, catalog, volume, soft, t_last, time, prev, cap, 0, tau)
            rates, indices, total = OK.compute_rates(Q, 1.0, T, nu0, cascade_mode=False)
            if total > 0:
                t_wait = -np.log(draws.u_wait()) / total
                if t_wait < remaining:
                    time += t_wait
                    eps_macro += unit * (strain_rate * t_wait)
                    remaining -= t_wait
                    k = OK.select_event(rates, total, draws.u_sel())
                    if k == -1:
                        continue
                    x, y, z, m = OK.decode_index_3d(int(indices[k]), ny, nz, M)
                    C = catalog[x, y, z, m].copy()
                    OK.apply_flip_3d(eps_p, soft, t_last, catalog, x, y, z, m, time, jp, jt, cap, jn)
                    prev[x, y, z] = C
                    catalog[x, y, z] = draws.catalog(M)
                    Q0[x, y, z] = draws.q0(M)
                    sig = update_stresses()
                    events.append((x, y, z, m, time))
                    if max_events is not None and len(events) >= max_events:
                        return result()
                    continue
            eps_macro += unit * (strain_rate * remaining)
            time += remaining
            remaining = 0.0
        sig = update_stresses()
        for _ in range(mixed_max_iter):
            sm = sig.mean(axis=(0, 1, 2))
            err = np.zeros((3, 3))
            err_max = 0.0
            for idx, target in stress_targets.items():
                e = target - sm[idx]
                err[idx] = e
                err_max = max(err_max, abs(e))
            if err_max < mixed_tol:
                break
            corr = (err - nu_avg * np.trace(err) * np.eye(3)) / E_avg
            corr[tuple(component)] = 0.0
            eps_macro += corr
            sig = update_stresses()
        steps_done += 1
    return result()
