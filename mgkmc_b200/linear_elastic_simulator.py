"""Drop-in small-strain LS solvers backed by the CUDA library.

``spectral_solver_2d`` keeps the signature and return value of
mgkmc/linear_elastic_simulator.py:12-88 (numpy in, numpy out); the work runs
on the current CUDA device through ``mgk_ls2d_*``.  ``Ls2dSolver`` is the
device-resident interface (torch CUDA tensors in and out, plan reused across
calls) that the KMC driver and the serving layer use.

The ``Gamma`` argument is accepted for signature compatibility and ignored:
the Green operator is evaluated on the fly from the mean moduli, which is how
the reference builds it whenever it is not passed (:25-29) and how its own
drivers build it when they pass it (:142-145).
"""
import ctypes
import threading

import numpy as np

from . import _lib as L

_PLANE = {"plane_strain": L.PLANE_STRAIN, "plane_stress": L.PLANE_STRESS}


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("mgkmc_b200 needs a CUDA device (no CPU fallback)")
    return torch


class Ls2dBatch:
    """Plan-owning batch of 2D LS replicas ("slots") on one device.

    ``sizes`` lists each replica's (nx, ny); sizes may differ.  Fields are
    torch float64 CUDA tensors in the reference layouts: E, nu (nx, ny);
    eps_plastic, eps, sig (nx, ny, 2, 2).  ``precision`` is "fp64" (the
    reference's arithmetic) or "mixed" (FP32 bulk iterations, FP64 finish)."""

    def __init__(self, sizes, plane_mode="plane_strain", precision="fp64", device=None):
        torch = _torch()
        self.sizes = [(int(a), int(b)) for a, b in sizes]
        self.nrep = len(self.sizes)
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.plane_mode = plane_mode
        self.precision = precision
        nx = (ctypes.c_int * self.nrep)(*[a for a, _ in self.sizes])
        ny = (ctypes.c_int * self.nrep)(*[b for _, b in self.sizes])
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            L.check(L.lib().mgk_ls2d_create_batch(self.nrep, nx, ny, _PLANE[plane_mode],
                                                  L.FP64 if precision == "fp64" else L.MIXED, ctypes.byref(h)),
                    "mgk_ls2d_create_batch")
        self._h = h
        self._keep = {}
        self.infos = (L.LsInfo * self.nrep)()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                L.lib().mgk_ls2d_destroy(h)
            except Exception:
                pass
            self._h = None

    def set_material(self, rep, E, nu, eps_plastic=None, stream=None):
        self._keep[("m", rep)] = (E, nu, eps_plastic)  # alive until the stream has consumed them
        L.check(L.lib().mgk_ls2d_set_material_rep(self._h, int(rep), L.ptr(E), L.ptr(nu), L.ptr(eps_plastic),
                                                  L.stream_ptr(stream)), "mgk_ls2d_set_material")

    def set_eigenstrain(self, rep, eps_plastic, stream=None):
        self._keep[("e", rep)] = eps_plastic
        L.check(L.lib().mgk_ls2d_set_eigenstrain_rep(self._h, int(rep), L.ptr(eps_plastic), L.stream_ptr(stream)),
                "mgk_ls2d_set_eigenstrain")

    def set_lame(self, rep, lam, mu, eps_plastic=None, stream=None):
        """Lame fields given directly (the secant solver's inputs); reference
        medium (mean lam, mean mu)."""
        self._keep[("m", rep)] = (lam, mu, eps_plastic)
        L.check(L.lib().mgk_ls2d_set_lame_rep(self._h, int(rep), L.ptr(lam), L.ptr(mu), L.ptr(eps_plastic),
                                              L.stream_ptr(stream)), "mgk_ls2d_set_lame")

    def set_secant(self, d, k):
        """Secant degradation law for every replica (d = 0: linear); FP64 plans."""
        L.check(L.lib().mgk_ls2d_set_secant(self._h, float(d), float(k)), "mgk_ls2d_set_secant")

    def set_rose(self, eta, mu_floor_fraction=0.1, plane_mode="plane_strain"):
        """Rose secant-modulus law for every replica; call before set_lame (the
        reference medium depends on the floor); FP64 plans."""
        L.check(L.lib().mgk_ls2d_set_rose(self._h, float(eta), float(mu_floor_fraction),
                                          1 if plane_mode == "plane_stress" else 0), "mgk_ls2d_set_rose")

    def set_landau(self, v, capping=0, e_cap=0.0, tangent_ratio=0.1, smooth_power=1.0, plane_stress=False):
        """Landau law for every replica: v = (v1, v2, v3, g1, g2, g3, g4);
        capping 0 none, 1 piecewise, 2 smooth at e_cap; plane_stress solves
        e33 per voxel (sigma33 = 0); FP64 plans."""
        arr = (ctypes.c_double * 7)(*[float(a) for a in v])
        L.check(L.lib().mgk_ls2d_set_landau(self._h, ctypes.cast(arr, ctypes.c_void_p), int(capping), float(e_cap),
                                            float(tangent_ratio), float(smooth_power), 1 if plane_stress else 0),
                "mgk_ls2d_set_landau")

    def set_e33_out(self, rep, e33):
        """Device buffer (N doubles) for replica rep's plane-stress Landau e33
        in later solves (None: not written)."""
        self._keep[("e33", rep)] = e33
        L.check(L.lib().mgk_ls2d_set_e33_out(self._h, int(rep), L.ptr(e33)), "mgk_ls2d_set_e33_out")

    def set_anderson(self, m):
        """Type-II Anderson mixing of depth m (0: off) inside the device loop of
        later solves; FP64 plans, one replica per solve."""
        L.check(L.lib().mgk_ls2d_set_anderson(self._h, int(m)), "mgk_ls2d_set_anderson")

    def solve(self, reps, eps_bars, eps_out, sig_out, eps_init=None, max_iter=200, tol=1e-6, sync=True,
              stream=None):
        """Solve replicas ``reps`` (one launch per stage for all of them).
        eps_bars: sequence of (2,2); eps_out/sig_out/eps_init: sequences of
        tensors (or None entries).  Returns the list of LsInfo when sync."""
        n = len(reps)
        sel = (ctypes.c_int * n)(*[int(r) for r in reps])
        eb = (ctypes.c_double * (4 * n))(*np.concatenate([np.asarray(e, dtype=np.float64).reshape(4)
                                                           for e in eps_bars]))
        P = ctypes.c_void_p

        def parr(ts):
            if ts is None:
                return None
            return (P * n)(*[None if t is None else t.data_ptr() for t in ts])

        infos = (L.LsInfo * n)() if sync else None
        st = L.lib().mgk_ls2d_solve_batch(self._h, n, sel, eb, parr(eps_init), parr(eps_out), parr(sig_out),
                                          int(max_iter), float(tol), infos, L.stream_ptr(stream))
        L.check(st, "mgk_ls2d_solve_batch", allow=(L.OK, L.NONFINITE))
        return list(infos) if sync else None

    def autotune(self, reps, eps_bars, n=5, stream=None):
        """Times every kernel family that can serve this plan on the selection
        and keeps the fastest; returns (family, ms per iteration): 0 for the
        CTA-wide passes, 256/512/1024 for the warp-line kernels.  Replicas must
        have their material; their iterates are left unspecified."""
        k = len(reps)
        sel = (ctypes.c_int * k)(*[int(r) for r in reps])
        eb = (ctypes.c_double * (4 * k))(*np.concatenate([np.asarray(e, dtype=np.float64).reshape(4)
                                                           for e in eps_bars]))
        ch, ms = ctypes.c_int(), ctypes.c_float()
        L.check(L.lib().mgk_ls2d_autotune(self._h, k, sel, eb, int(n), ctypes.byref(ch), ctypes.byref(ms),
                                          L.stream_ptr(stream)), "mgk_ls2d_autotune")
        self.family = ch.value
        return ch.value, ms.value

    def set_family(self, family):
        """Kernel family (0 CTA-wide, 256/512/1024 warp-line), e.g. one chosen
        by ``autotune`` for an equal plan."""
        L.check(L.lib().mgk_ls2d_set_family(self._h, int(family)), "mgk_ls2d_set_family")
        self.family = int(family)

    def collect(self, reps, stream=None):
        """LsInfo of the last solve of ``reps`` after ``solve(..., sync=False)``
        (one synchronisation of the stream)."""
        n = len(reps)
        sel = (ctypes.c_int * n)(*[int(r) for r in reps])
        infos = (L.LsInfo * n)()
        st = L.lib().mgk_ls2d_collect(self._h, n, sel, infos, L.stream_ptr(stream))
        L.check(st, "mgk_ls2d_collect", allow=(L.OK, L.NONFINITE))
        return list(infos)

    def profile_kernels(self, reps, eps_bars, fp32=False, n=50, stream=None):
        """Mean (row_ms, col_ms) of the two iteration kernels over the
        selection (CUDA events on the stream)."""
        k = len(reps)
        sel = (ctypes.c_int * k)(*[int(r) for r in reps])
        eb = (ctypes.c_double * (4 * k))(*np.concatenate([np.asarray(e, dtype=np.float64).reshape(4)
                                                           for e in eps_bars]))
        r, c = ctypes.c_float(), ctypes.c_float()
        L.check(L.lib().mgk_ls2d_profile_batch(self._h, k, sel, eb, 1 if fp32 else 0, int(n), ctypes.byref(r),
                                               ctypes.byref(c), L.stream_ptr(stream)), "mgk_ls2d_profile_batch")
        return r.value, c.value


class Ls2dSolver(Ls2dBatch):
    """One-replica plan with the single-solve interface."""

    def __init__(self, nx, ny, plane_mode="plane_strain", precision="fp64", device=None):
        super().__init__([(nx, ny)], plane_mode, precision, device)
        self.nx, self.ny = int(nx), int(ny)

    def set_material(self, E, nu, eps_plastic=None, stream=None):
        super().set_material(0, E, nu, eps_plastic, stream)

    def set_eigenstrain(self, eps_plastic, stream=None):
        super().set_eigenstrain(0, eps_plastic, stream)

    def solve(self, eps_bar, eps_out, sig_out, eps_init=None, max_iter=200, tol=1e-6, sync=True, stream=None):
        infos = super().solve([0], [eps_bar], [eps_out], [sig_out], None if eps_init is None else [eps_init],
                              max_iter, tol, sync, stream)
        return infos[0] if sync else None

    def profile_kernels(self, eps_bar, reps=50, stream=None):
        return super().profile_kernels([0], [eps_bar], False, reps, stream)


_PLANS = {}


def _plan(nx, ny, plane_mode, device_index):
    key = (nx, ny, plane_mode, device_index)
    p = _PLANS.get(key)
    if p is None:
        p = Ls2dSolver(nx, ny, plane_mode)
        _PLANS[key] = p
    return p


def spectral_solver_2d(E, nu, eps_bar, eps_plastic=None, max_iter=200, tol=1e-6, verbose=False, pixel=1.0,
                       plane_mode="plane_strain", Gamma=None, eps_init=None):
    """Single-point 2D Lippmann-Schwinger solve (linear_elastic_simulator.py:12-88).

    Returns (eps, sig, eps.mean(axis=(0,1)), sig.mean(axis=(0,1))) as numpy
    float64 arrays.  ``verbose``, ``pixel`` and ``Gamma`` do not change the
    result (pixel cancels in the Green operator)."""
    torch = _torch()
    E = np.ascontiguousarray(E, dtype=np.float64)
    nu = np.ascontiguousarray(nu, dtype=np.float64)
    nx, ny = E.shape
    dev = torch.device("cuda", torch.cuda.current_device())
    p = _plan(nx, ny, plane_mode, dev.index)
    tE = torch.from_numpy(E).to(dev, non_blocking=False)
    tnu = torch.from_numpy(nu).to(dev)
    tep = None if eps_plastic is None else torch.from_numpy(np.ascontiguousarray(eps_plastic, dtype=np.float64)).to(dev)
    tin = None if eps_init is None else torch.from_numpy(np.ascontiguousarray(eps_init, dtype=np.float64)).to(dev)
    eps = torch.empty((nx, ny, 2, 2), dtype=torch.float64, device=dev)
    sig = torch.empty_like(eps)
    p.set_material(tE, tnu, tep)
    info = p.solve(eps_bar, eps, sig, eps_init=tin, max_iter=max_iter, tol=tol, sync=True)
    if verbose:
        print(f"LS 2D: {info.iterations} iterations, diff = {info.final_diff:.3e}")
    eps_np = eps.cpu().numpy()
    sig_np = sig.cpu().numpy()
    return eps_np, sig_np, eps_np.mean(axis=(0, 1)), sig_np.mean(axis=(0, 1))


_PLANS_SECANT = {}


def spectral_solver_secant_2d(lam, mu, d, k, eps_bar, eps_plastic=None, max_iter=400, tol=1e-6, verbose=False,
                              pixel=1.0, plane_mode="plane_strain", Gamma=None, eps_init=None):
    """Nonlinear 2D Lippmann-Schwinger solve with the secant degradation law
    (linear_elastic_simulator.py:614-765): sigma = lam tr(e) I + 2 mu_sec e,
    e = eps - eps_plastic, mu_sec = mu (1 - d (1 - exp(-k eps_eq(e)))), the
    reference medium (mean lam, mean mu) held fixed.  ``lam`` is the caller's
    (effective, for plane stress) lambda field, as in the reference.  Returns
    (eps, sig, eps.mean(axis=(0,1)), sig.mean(axis=(0,1)))."""
    torch = _torch()
    lam = np.array(np.broadcast_to(np.asarray(lam, dtype=np.float64), np.shape(mu) or np.shape(lam)))
    mu = np.array(np.broadcast_to(np.asarray(mu, dtype=np.float64), lam.shape))
    nx, ny = lam.shape
    dev = torch.device("cuda", torch.cuda.current_device())
    key = (nx, ny, dev.index)
    p = _PLANS_SECANT.get(key)
    if p is None:
        p = _PLANS_SECANT[key] = Ls2dBatch([(nx, ny)])
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(dev)
    eps = torch.empty((nx, ny, 2, 2), dtype=torch.float64, device=dev)
    sig = torch.empty_like(eps)
    p.set_lame(0, t(lam), t(mu), None if eps_plastic is None else t(eps_plastic))
    p.set_secant(d, k)
    info = p.solve([0], [eps_bar], [eps], [sig], eps_init=None if eps_init is None else [t(eps_init)],
                   max_iter=max_iter, tol=tol)[0]
    if verbose:
        print(f"secant LS 2D: {info.iterations} iterations, diff = {info.final_diff:.3e}")
    eps_np = eps.cpu().numpy()
    sig_np = sig.cpu().numpy()
    return eps_np, sig_np, eps_np.mean(axis=(0, 1)), sig_np.mean(axis=(0, 1))


_PLANS_ROSE = {}


def spectral_solver_rose_2d(lam, mu, eta, mu_floor_fraction=0.1, eps_bar=None, eps_plastic=None, max_iter=400,
                            tol=1e-6, verbose=False, pixel=1.0, plane_mode="plane_strain", Gamma=None,
                            eps_init=None):
    """Nonlinear 2D Lippmann-Schwinger solve with the Rose secant-modulus law
    (linear_elastic_simulator.py:852-950): G = max(mu exp(-eta eps_eq),
    floor mu) at constant bulk modulus, reference medium (mean lam,
    (mean mu + floor mean mu) / 2).  ``lam`` is the 3D Lame lambda (plane
    stress is reduced per voxel, as in the reference).  Macro strain,
    eigenstrain and warm start must be symmetric (the strain's [0,1] entry
    drives the law).  Returns (eps, sig, eps.mean(axis=(0,1)),
    sig.mean(axis=(0,1)))."""
    torch = _torch()
    lam = np.array(np.broadcast_to(np.asarray(lam, dtype=np.float64), np.shape(mu) or np.shape(lam)))
    mu = np.array(np.broadcast_to(np.asarray(mu, dtype=np.float64), lam.shape))
    eps_bar = np.asarray(eps_bar, dtype=np.float64)
    for a in (eps_bar, eps_plastic, eps_init):
        if a is not None and not np.array_equal(np.asarray(a)[..., 0, 1], np.asarray(a)[..., 1, 0]):
            raise NotImplementedError("spectral_solver_rose_2d: asymmetric strain tensors are not supported")
    nx, ny = lam.shape
    dev = torch.device("cuda", torch.cuda.current_device())
    key = (nx, ny, dev.index)
    p = _PLANS_ROSE.get(key)
    if p is None:
        p = _PLANS_ROSE[key] = Ls2dBatch([(nx, ny)])
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(dev)
    eps = torch.empty((nx, ny, 2, 2), dtype=torch.float64, device=dev)
    sig = torch.empty_like(eps)
    p.set_rose(eta, mu_floor_fraction, plane_mode)
    p.set_lame(0, t(lam), t(mu), None if eps_plastic is None else t(eps_plastic))
    info = p.solve([0], [eps_bar], [eps], [sig], eps_init=None if eps_init is None else [t(eps_init)],
                   max_iter=max_iter, tol=tol)[0]
    if verbose:
        print(f"Rose LS 2D: {info.iterations} iterations, diff = {info.final_diff:.3e}")
    eps_np = eps.cpu().numpy()
    sig_np = sig.cpu().numpy()
    return eps_np, sig_np, eps_np.mean(axis=(0, 1)), sig_np.mean(axis=(0, 1))


_PLANS_LANDAU = {}
_PLANS_LANDAU_LOCK = threading.Lock()


def spectral_solver_landau_2d(lam, mu, v1, v2, v3, g1, g2, g3, g4, eps_bar, eps_plastic=None, max_iter=400, tol=1e-6,
                              verbose=False, pixel=1.0, plane_mode="plane_strain", Gamma=None, eps_init=None,
                              strain_capping_enabled=False, strain_capping_limit=None,
                              strain_capping_tangent_ratio=0.1, strain_capping_type="piecewise",
                              strain_capping_smooth_power=1.0, solver="dbfft", e33_state=None, anderson_m=5):
    """Nonlinear 2D Lippmann-Schwinger solve with the Landau small-strain law
    (linear_elastic_simulator.py:952-1228, solver "dbfft"), plane strain or
    plane stress (e33 per voxel from the law's Newton solve of sigma33 = 0;
    ``e33_state``, when given, receives the final e33 field as the
    reference's does; its warm start is not needed, each evaluation solving
    e33 to convergence): the basic scheme with the (mean lam, mean mu) medium
    and type-II Anderson mixing of the last anderson_m iterates, the whole
    loop (update norm, convergence decision, least-squares fit and mix) on
    the device in one graph launch.  Returns (eps, sig, eps.mean(axis=(0,1)),
    sig.mean(axis=(0,1))); a non-finite update raises FloatingPointError as
    the reference does.  The Newton-CG branch and asymmetric strains are not
    built (NotImplementedError); anderson_m is limited to 8."""
    if plane_mode not in ("plane_strain", "plane_stress"):
        raise ValueError(f"spectral_solver_landau_2d: plane_mode={plane_mode!r}")
    if solver != "dbfft":
        raise NotImplementedError("spectral_solver_landau_2d: only the basic scheme (solver='dbfft') is built")
    m = int(anderson_m)
    if m < 0 or m > 8:
        raise NotImplementedError("spectral_solver_landau_2d: anderson_m must be 0..8")
    torch = _torch()
    lam = np.array(np.broadcast_to(np.asarray(lam, dtype=np.float64), np.shape(mu) or np.shape(lam)))
    mu = np.array(np.broadcast_to(np.asarray(mu, dtype=np.float64), lam.shape))
    eps_bar = np.asarray(eps_bar, dtype=np.float64)
    for a in (eps_bar, eps_plastic, eps_init):
        if a is not None and not np.array_equal(np.asarray(a)[..., 0, 1], np.asarray(a)[..., 1, 0]):
            raise NotImplementedError("spectral_solver_landau_2d: asymmetric strain tensors are not supported")
    cap, e_cap = 0, 0.0
    if strain_capping_enabled:
        cap = 2 if strain_capping_type == "smooth" else 1
        if strain_capping_limit is None or strain_capping_limit <= 0:
            e_cap = float(np.sqrt(0.2 * mu.mean() / abs(g4))) if g4 < 0 else 999.0
        else:
            e_cap = float(strain_capping_limit)
    nx, ny = lam.shape
    dev = torch.device("cuda", torch.cuda.current_device())
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(dev)
    with _PLANS_LANDAU_LOCK:
        key = (nx, ny, dev.index)
        p = _PLANS_LANDAU.get(key)
        if p is None:
            p = _PLANS_LANDAU[key] = Ls2dBatch([(nx, ny)])
        ps = plane_mode == "plane_stress"
        p.set_landau((v1, v2, v3, g1, g2, g3, g4), cap, e_cap, strain_capping_tangent_ratio,
                     strain_capping_smooth_power, plane_stress=ps)
        p.set_anderson(m)
        p.set_lame(0, t(lam), t(mu), None if eps_plastic is None else t(eps_plastic))
        eps = torch.empty((nx, ny, 2, 2), dtype=torch.float64, device=dev)
        sig = torch.empty_like(eps)
        e33 = torch.empty((nx, ny), dtype=torch.float64, device=dev) if ps and e33_state is not None else None
        p.set_e33_out(0, e33)
        init = None if eps_init is None else [t(eps_init)]
        try:
            info = p.solve([0], [eps_bar], [eps], [sig], eps_init=init, max_iter=max_iter, tol=tol)[0]
        finally:
            p.set_e33_out(0, None)
        eps_np, sig_np = eps.cpu().numpy(), sig.cpu().numpy()
        if e33 is not None:
            e33_state["e33"] = e33.cpu().numpy()
    if info.status == L.NONFINITE or not np.isfinite(info.final_diff):
        raise FloatingPointError("spectral_solver_landau_2d: non-finite strain update in LS loop (Landau energy "
                                 "likely unstable at this strain; consider strain capping or smaller load steps).")
    if verbose:
        print(f"  [landau-LS] {info.iterations} iterations: rel_diff = {info.final_diff:.3e}")
    return eps_np, sig_np, eps_np.mean(axis=(0, 1)), sig_np.mean(axis=(0, 1))


class Ls3dBatch:
    """Plan-owning batch of 3D LS replicas.  Fields: E, nu (nx,ny,nz);
    eps_plastic, eps, sig (nx,ny,nz,3,3) torch float64 CUDA tensors.
    ``precision``: "fp64", or "mixed" (FP32 phase then FP64; every side 64, 96
    or 128)."""

    def __init__(self, sizes, device=None, precision="fp64"):
        torch = _torch()
        self.sizes = [tuple(int(v) for v in s) for s in sizes]
        self.nrep = len(self.sizes)
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        nx = (ctypes.c_int * self.nrep)(*[s[0] for s in self.sizes])
        ny = (ctypes.c_int * self.nrep)(*[s[1] for s in self.sizes])
        nz = (ctypes.c_int * self.nrep)(*[s[2] for s in self.sizes])
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            L.check(L.lib().mgk_ls3d_create_batch(self.nrep, nx, ny, nz, ctypes.byref(h)), "mgk_ls3d_create_batch")
        self._h = h
        self._keep = {}
        self.precision = precision
        if precision != "fp64":
            L.check(L.lib().mgk_ls3d_set_precision(h, L.MIXED), "mgk_ls3d_set_precision")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                L.lib().mgk_ls3d_destroy(h)
            except Exception:
                pass
            self._h = None

    def set_material(self, rep, E, nu, eps_plastic=None, stream=None):
        self._keep[("m", rep)] = (E, nu, eps_plastic)
        L.check(L.lib().mgk_ls3d_set_material_rep(self._h, int(rep), L.ptr(E), L.ptr(nu), L.ptr(eps_plastic),
                                                  L.stream_ptr(stream)), "mgk_ls3d_set_material")

    def set_lame(self, rep, lam, mu, eps_plastic=None, stream=None):
        """Lame fields given directly, medium (mean lam, mean mu): the secant
        solver's inputs (linear_elastic_simulator.py:768-784)."""
        self._keep[("m", rep)] = (lam, mu, eps_plastic)
        L.check(L.lib().mgk_ls3d_set_lame_rep(self._h, int(rep), L.ptr(lam), L.ptr(mu), L.ptr(eps_plastic),
                                              L.stream_ptr(stream)), "mgk_ls3d_set_lame")

    def set_secant(self, d, k):
        """Secant degradation law for every replica (0 < d <= 1; d = 0 linear)."""
        L.check(L.lib().mgk_ls3d_set_secant(self._h, float(d), float(k)), "mgk_ls3d_set_secant")

    def set_landau(self, v, capping=0, e_cap=0.0, tangent_ratio=0.1, smooth_power=1.0):
        """Landau law for every replica: v = (v1, v2, v3, g1, g2, g3, g4);
        capping 0 none, 1 piecewise, 2 smooth at e_cap; FP64 plans."""
        arr = (ctypes.c_double * 7)(*[float(a) for a in v])
        L.check(L.lib().mgk_ls3d_set_landau(self._h, ctypes.cast(arr, ctypes.c_void_p), int(capping), float(e_cap),
                                            float(tangent_ratio), float(smooth_power)), "mgk_ls3d_set_landau")

    def set_eigenstrain(self, rep, eps_plastic, stream=None):
        self._keep[("e", rep)] = eps_plastic
        L.check(L.lib().mgk_ls3d_set_eigenstrain_rep(self._h, int(rep), L.ptr(eps_plastic), L.stream_ptr(stream)),
                "mgk_ls3d_set_eigenstrain")

    def solve(self, reps, eps_bars, eps_out, sig_out, eps_init=None, max_iter=200, tol=1e-6, sync=True,
              stream=None):
        n = len(reps)
        sel = (ctypes.c_int * n)(*[int(r) for r in reps])
        eb = (ctypes.c_double * (9 * n))(*np.concatenate([np.asarray(e, dtype=np.float64).reshape(9)
                                                           for e in eps_bars]))
        P = ctypes.c_void_p

        def parr(ts):
            return None if ts is None else (P * n)(*[None if t is None else t.data_ptr() for t in ts])

        infos = (L.LsInfo3 * n)() if sync else None
        st = L.lib().mgk_ls3d_solve_batch(self._h, n, sel, eb, parr(eps_init), parr(eps_out), parr(sig_out),
                                          int(max_iter), float(tol), infos, L.stream_ptr(stream))
        L.check(st, "mgk_ls3d_solve_batch", allow=(L.OK, L.NONFINITE))
        return list(infos) if sync else None


_PLANS3 = {}


def spectral_solver_3d(E, nu, eps_bar, eps_plastic=None, max_iter=200, tol=1e-6, verbose=False, pixel=1.0,
                       Gamma=None, eps_init=None):
    """3D Lippmann-Schwinger solve (linear_elastic_simulator.py:274-376);
    numpy in/out, same returns as the reference."""
    torch = _torch()
    E = np.ascontiguousarray(E, dtype=np.float64)
    nu = np.ascontiguousarray(nu, dtype=np.float64)
    shape = E.shape
    dev = torch.device("cuda", torch.cuda.current_device())
    key = (shape, dev.index)
    p = _PLANS3.get(key)
    if p is None:
        p = _PLANS3[key] = Ls3dBatch([shape])
    tep = None if eps_plastic is None else torch.from_numpy(np.ascontiguousarray(eps_plastic, dtype=np.float64)).to(dev)
    tin = None if eps_init is None else torch.from_numpy(np.ascontiguousarray(eps_init, dtype=np.float64)).to(dev)
    eps = torch.empty(shape + (3, 3), dtype=torch.float64, device=dev)
    sig = torch.empty_like(eps)
    p.set_material(0, torch.from_numpy(E).to(dev), torch.from_numpy(nu).to(dev), tep)
    info = p.solve([0], [eps_bar], [eps], [sig], None if tin is None else [tin], max_iter, tol)[0]
    if verbose:
        print(f"LS 3D: {info.iterations} iterations, diff = {info.final_diff:.3e}")
    e, s = eps.cpu().numpy(), sig.cpu().numpy()
    return e, s, e.mean(axis=(0, 1, 2)), s.mean(axis=(0, 1, 2))


_PLANS3_SECANT = {}


def spectral_solver_secant_3d(lam, mu, d, k, eps_bar, eps_plastic=None, max_iter=400, tol=1e-6, verbose=False,
                              pixel=1.0, Gamma=None, eps_init=None):
    """Nonlinear 3D Lippmann-Schwinger solve with the secant degradation law
    (linear_elastic_simulator.py:768-850): sigma = lam tr(e) I + 2 mu_sec e,
    e = eps - eps_plastic, mu_sec = mu (1 - d (1 - exp(-k eps_eq(e)))), the
    reference medium (mean lam, mean mu) held fixed.  Returns
    (eps, sig, eps.mean(axis=(0,1,2)), sig.mean(axis=(0,1,2)))."""
    torch = _torch()
    lam = np.array(np.broadcast_to(np.asarray(lam, dtype=np.float64), np.shape(mu) or np.shape(lam)))
    mu = np.array(np.broadcast_to(np.asarray(mu, dtype=np.float64), lam.shape))
    shape = lam.shape
    dev = torch.device("cuda", torch.cuda.current_device())
    key = (shape, dev.index)
    p = _PLANS3_SECANT.get(key)
    if p is None:
        p = _PLANS3_SECANT[key] = Ls3dBatch([shape])
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(dev)
    eps = torch.empty(shape + (3, 3), dtype=torch.float64, device=dev)
    sig = torch.empty_like(eps)
    p.set_lame(0, t(lam), t(mu), None if eps_plastic is None else t(eps_plastic))
    p.set_secant(d, k)
    info = p.solve([0], [eps_bar], [eps], [sig], None if eps_init is None else [t(eps_init)], max_iter, tol)[0]
    if verbose:
        print(f"secant LS 3D: {info.iterations} iterations, diff = {info.final_diff:.3e}")
    e, s_ = eps.cpu().numpy(), sig.cpu().numpy()
    return e, s_, e.mean(axis=(0, 1, 2)), s_.mean(axis=(0, 1, 2))


_PLANS3_LANDAU = {}


def spectral_solver_landau_3d(lam, mu, v1, v2, v3, g1, g2, g3, g4, eps_bar, eps_plastic=None, max_iter=400, tol=1e-6,
                              verbose=False, pixel=1.0, Gamma=None, eps_init=None, strain_capping_enabled=False,
                              strain_capping_limit=None, strain_capping_tangent_ratio=0.1,
                              strain_capping_type="piecewise", strain_capping_smooth_power=1.0, solver="dbfft"):
    """Nonlinear 3D Lippmann-Schwinger solve with the Landau small-strain law
    (linear_elastic_simulator.py:1231-1350): the basic scheme with the (mean
    lam, mean mu) medium, the whole loop on the device (the law compiled into
    the z-line and output kernels).  Returns (eps, sig, eps.mean(axis=(0,1,2)),
    sig.mean(axis=(0,1,2))); a non-finite update raises FloatingPointError as
    the reference does.  Symmetric strain tensors only."""
    if solver == "newton_cg":
        raise NotImplementedError("Newton-CG solver is not yet implemented for 3D small-strain")
    torch = _torch()
    lam = np.array(np.broadcast_to(np.asarray(lam, dtype=np.float64), np.shape(mu) or np.shape(lam)))
    mu = np.array(np.broadcast_to(np.asarray(mu, dtype=np.float64), lam.shape))
    eps_bar = np.asarray(eps_bar, dtype=np.float64)
    for a in (eps_bar, eps_plastic, eps_init):
        if a is not None and not np.array_equal(np.asarray(a), np.swapaxes(np.asarray(a), -1, -2)):
            raise NotImplementedError("spectral_solver_landau_3d: asymmetric strain tensors are not supported")
    cap, e_cap = 0, 0.0
    if strain_capping_enabled:
        cap = 2 if strain_capping_type == "smooth" else 1
        if strain_capping_limit is None or strain_capping_limit <= 0:
            e_cap = float(np.sqrt(0.2 * mu.mean() / abs(g4))) if g4 < 0 else 999.0
        else:
            e_cap = float(strain_capping_limit)
    shape = lam.shape
    dev = torch.device("cuda", torch.cuda.current_device())
    key = (shape, dev.index)
    p = _PLANS3_LANDAU.get(key)
    if p is None:
        p = _PLANS3_LANDAU[key] = Ls3dBatch([shape])
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(dev)
    p.set_lame(0, t(lam), t(mu), None if eps_plastic is None else t(eps_plastic))
    p.set_landau((v1, v2, v3, g1, g2, g3, g4), cap, e_cap, strain_capping_tangent_ratio, strain_capping_smooth_power)
    eps = torch.empty(shape + (3, 3), dtype=torch.float64, device=dev)
    sig = torch.empty_like(eps)
    info = p.solve([0], [eps_bar], [eps], [sig], None if eps_init is None else [t(eps_init)], max_iter, tol)[0]
    if info.status == L.NONFINITE or not np.isfinite(info.final_diff):
        raise FloatingPointError("spectral_solver_landau_3d: non-finite strain update in LS loop (Landau energy "
                                 "likely unstable at this strain; consider strain capping or smaller load steps).")
    if verbose:
        print(f"landau LS 3D: {info.iterations} iterations, diff = {info.final_diff:.3e}")
    e, s_ = eps.cpu().numpy(), sig.cpu().numpy()
    return e, s_, e.mean(axis=(0, 1, 2)), s_.mean(axis=(0, 1, 2))


def update_stress_fft_full(eps_plastic_field, eps_macro, E, nu, pixel=1.0, max_iter=200, tol=1e-6, verbose=False):
    """mgkmc/stz/update_fft.py:4-22: the 3D solve with an eigenstrain field."""
    return spectral_solver_3d(E, nu, eps_macro, eps_plastic=eps_plastic_field, max_iter=max_iter, tol=tol,
                              verbose=verbose, pixel=pixel)


# ------------------------------------------------ mixed-BC load ramps ---
_COMP_LABELS = {(0, 0): "xx", (1, 1): "yy", (2, 2): "zz", (0, 1): "xy", (0, 2): "xz", (1, 2): "yz", (1, 0): "yx",
                (2, 0): "zx", (2, 1): "zy"}


def _vtk_step(ival, path, s, eps, sig, E, nu, pixel):
    """The ramps' per-step VTK file (linear_elastic_simulator.py:237-246):
    ival "current" rewrites <path>.vtu, an integer writes <path>_<step>.vtu
    every ival steps; "none", "last" and None write nothing here."""
    if ival is None or ival in ("none", "last"):
        return
    from .vtk import export_to_vtk
    if ival == "current":
        export_to_vtk(f"{path}.vtu", eps, sig, E, nu, pixel, match_matplotlib_orientation=True)
    elif isinstance(ival, int) and s % ival == 0:
        export_to_vtk(f"{path}_{s:06d}.vtu", eps, sig, E, nu, pixel, match_matplotlib_orientation=True)


def _vtk_final(ival, path, n_steps, eps, sig, E, nu, pixel):
    """The ramps' final VTK file (:253-256): <path>_final.vtu for "last", or
    for an integer interval that did not end on the last step."""
    if ival == "last" or (isinstance(ival, int) and n_steps % ival != 0):
        from .vtk import export_to_vtk
        export_to_vtk(f"{path}_final.vtu", eps, sig, E, nu, pixel, match_matplotlib_orientation=True)


def _ramp(dim, E, nu, target_strain_mask, target_values, n_steps, pixel, tol_ls, max_iter_ls, tol_macro,
          max_iter_macro, store, plane_mode, log_path, global_log_path, driving_component, enable_console, vtk_path,
          vtk_interval, solver_kw):
    """Mixed stress/strain load ramp of linear_elastic_simulation_2d/3d
    (linear_elastic_simulator.py:90-272 / :378-566) on one device-resident LS
    plan: targets ramped linearly over n_steps + 1 load steps; per load step
    the macro loop (:176-197) solves with the prescribed strain components,
    corrects the stress-controlled ones by the isotropic compliance
    (:150-152) until their mean-stress error is below tol_macro; every solve
    of a load step warm-starts from the previous load step's final field
    (:199).  Fields stay on the device between solves; only the stored
    fields and the per-step means come back."""
    import time as _time
    from datetime import datetime as _dt
    torch = _torch()
    chk_ival = solver_kw.pop("checkpoint_interval", None)
    chk_path = solver_kw.pop("checkpoint_path", "checkpoint")
    if chk_path and chk_ival not in (None, "none"):
        import os
        os.makedirs(os.path.dirname(chk_path) or ".", exist_ok=True)
    E = np.ascontiguousarray(E, dtype=np.float64)
    nu = np.ascontiguousarray(nu, dtype=np.float64)
    shape = E.shape
    mask = np.asarray(target_strain_mask, dtype=bool)
    target_values = np.asarray(target_values, dtype=np.float64)
    stress_mask = ~mask
    dev = torch.device("cuda", torch.cuda.current_device())
    plan = Ls2dBatch([shape], plane_mode=plane_mode) if dim == 2 else Ls3dBatch([shape])
    t = lambda a: torch.from_numpy(a).to(dev)
    plan.set_material(0, t(E), t(nu), None)
    E_avg, nu_avg = E.mean(), nu.mean()
    fshape = shape + (dim, dim)
    eps = torch.empty(fshape, dtype=torch.float64, device=dev)
    sig = torch.empty_like(eps)
    warm = torch.empty_like(eps)
    have_warm = False
    lbl = _COMP_LABELS.get(tuple(driving_component), "xx")
    log_f = open(log_path, "w", buffering=1) if log_path else None
    if log_f:
        hdr = f"{'Timestamp':<20} {'Elapsed(s)':<12} {'Step':<8} {'Eps_' + lbl:<14} {'Sig_' + lbl + '(GPa)':<16}\n"
        log_f.write(hdr)
        log_f.write("-" * len(hdr.rstrip()) + "\n")
    glog_f = open(global_log_path, "w", buffering=1) if global_log_path else None
    comps = [(0, 0), (1, 1), (0, 1)] if dim == 2 else [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]
    if glog_f:
        ghdr = f"{'GlobalStep':<12} " + " ".join(f"{'Eps_' + _COMP_LABELS[c]:<14}" for c in comps) + " " + \
               " ".join(f"{'Sig_' + _COMP_LABELS[c] + '(GPa)':<16}" for c in comps) + "\n"
        glog_f.write(ghdr)
        glog_f.write("-" * len(ghdr.rstrip()) + "\n")
    t0 = _time.time()
    eps_macro_list, sig_macro_list, eps_list, sig_list = [], [], [], []
    cur = np.zeros((dim, dim))
    axes = tuple(range(dim))
    for s in range(n_steps + 1):
        target_s = target_values * (s / n_steps)
        max_err = 0.0
        for _ in range(max_iter_macro):
            cur[mask] = target_s[mask]
            info = plan.solve([0], [cur], [eps], [sig], eps_init=[warm] if have_warm else None, max_iter=max_iter_ls,
                              tol=tol_ls)[0]
            sigM = np.array(info.sig_mean).reshape(dim, dim)
            err = np.zeros((dim, dim))
            err[stress_mask] = target_s[stress_mask] - sigM[stress_mask]
            max_err = np.max(np.abs(err[stress_mask])) if np.any(stress_mask) else 0.0
            if max_err < tol_macro:
                break
            d_eps = (err - nu_avg * np.trace(err) * np.eye(dim)) / E_avg
            cur[stress_mask] += d_eps[stress_mask]
        else:
            print(f"Warning: Macro loop did not converge at step {s} (err={max_err:.2e})")
        warm.copy_(eps)
        have_warm = True
        e_np, s_np = eps.cpu().numpy(), sig.cpu().numpy()
        epsM, sigM = e_np.mean(axis=axes), s_np.mean(axis=axes)
        eps_macro_list.append(epsM)
        sig_macro_list.append(sigM)
        if store:
            eps_list.append(e_np)
            sig_list.append(s_np)
        i, j = driving_component
        if enable_console:
            print(f"step {s}/{n_steps}: eps_{lbl}={epsM[i, j]:.4f}, sig_{lbl}={sigM[i, j] / 1e9:.4f} GPa")
        if log_f:
            log_f.write(f"{_dt.now().strftime('%Y-%m-%d %H:%M:%S'):<20} {_time.time() - t0:<12.3f} {s:<8} "
                        f"{epsM[i, j]:<14.6f} {sigM[i, j] / 1e9:<16.6f}\n")
        if glog_f:
            glog_f.write(f"{s:<12} " + " ".join(f"{epsM[c]:<14.6f}" for c in comps) + " " +
                         " ".join(f"{sigM[c] / 1e9:<16.6f}" for c in comps) + "\n")
        if chk_ival is not None and chk_ival not in ("none", "last"):
            name = None
            if chk_ival == "current":
                name = f"{chk_path}.h5"
            elif isinstance(chk_ival, int) and s % chk_ival == 0:
                name = f"{chk_path}_{s:06d}.h5"
            if name:
                _save_chk(dim, name, s, E, nu, e_np, s_np, epsM, sigM, pixel)
        _vtk_step(vtk_interval, vtk_path, s, e_np, s_np, E, nu, pixel)
    if chk_ival == "last" or (isinstance(chk_ival, int) and n_steps % chk_ival != 0):
        _save_chk(dim, f"{chk_path}_final.h5", n_steps, E, nu, e_np, s_np, epsM, sigM, pixel)
    _vtk_final(vtk_interval, vtk_path, n_steps, e_np, s_np, E, nu, pixel)
    total = _time.time() - t0
    m_, s_ = divmod(total, 60)
    h_, m_ = divmod(m_, 60)
    dur = (f"\nSimulation Finish Time: {_dt.now().strftime('%Y-%m-%d %H:%M:%S')}\nTotal Duration: {total:.2f} seconds "
           f"({int(h_):d}h {int(m_):02d}m {int(s_):02d}s)\n")
    if log_f:
        log_f.write(dur)
        log_f.close()
    if glog_f:
        glog_f.close()
    if enable_console:
        print(dur)
    return np.array(eps_macro_list), np.array(sig_macro_list), eps_list, sig_list


def _save_chk(dim, path, step, E, nu, eps, sig, epsM, sigM, pixel):
    from . import checkpoint as C
    if path.endswith(".h5") and not C._HAVE_H5PY:
        path = path[:-3]  # the .npz container of the same layout
    (C.save_checkpoint_2d if dim == 2 else C.save_checkpoint_3d)(path, step, E, nu, eps, sig, epsM, sigM, pixel)


def linear_elastic_simulation_2d(E, nu, target_strain_mask, target_values, n_steps=20, pixel=1.0, tol_ls=1e-6,
                                 max_iter_ls=200, tol_macro=1e-4, max_iter_macro=20, store=True,
                                 plane_mode="plane_strain", log_path=None, global_log_path=None,
                                 driving_component=(0, 0), enable_console=True, vtk_path=None, vtk_interval="none",
                                 **solver_kw):
    """Mixed stress/strain control in 2D (linear_elastic_simulator.py:90-272):
    returns (eps_macro (n_steps+1,2,2), sig_macro (n_steps+1,2,2), eps list,
    sig list).  Checkpoints (``checkpoint_interval``/``checkpoint_path``) use
    the reference's layout (``mgkmc_b200.checkpoint``)."""
    return _ramp(2, E, nu, target_strain_mask, target_values, n_steps, pixel, tol_ls, max_iter_ls, tol_macro,
                 max_iter_macro, store, plane_mode, log_path, global_log_path, driving_component, enable_console,
                 vtk_path, vtk_interval, dict(solver_kw))


def linear_elastic_simulation_3d(E, nu, target_strain_mask, target_values, n_steps=20, pixel=1.0, tol_ls=1e-6,
                                 max_iter_ls=200, tol_macro=1e-4, max_iter_macro=20, store=True, log_path=None,
                                 global_log_path=None, driving_component=(0, 0), enable_console=True, vtk_path=None,
                                 vtk_interval="none", **solver_kw):
    """Mixed stress/strain control in 3D (linear_elastic_simulator.py:378-566);
    returns as linear_elastic_simulation_2d with (…,3,3) tensors."""
    return _ramp(3, E, nu, target_strain_mask, target_values, n_steps, pixel, tol_ls, max_iter_ls, tol_macro,
                 max_iter_macro, store, "plane_strain", log_path, global_log_path, driving_component, enable_console,
                 vtk_path, vtk_interval, dict(solver_kw))


# ------------------------------------ nonlinear mixed-BC load ramps ---
# The load-step drivers of the secant, Rose and Landau solvers
# (linear_elastic_simulator.py:1353-2517).  Each load step runs the same
# macro loop as the linear ramps, calling the nonlinear device solver (the
# drop-ins above) once per macro iteration, warm-started from the previous
# load step's final field.  The stress-controlled components are corrected
# by the compliance of the solver's reference medium; the Landau ramps
# replace that slope per component by the secant slope of the last two macro
# iterates once it is trustworthy (:2186-2204).

def _vm_eq_2d(eps):
    """Von Mises equivalent strain of a 2D field with eps_33 = 0
    (elasticity.py:641-663): the in-plane trace removed, the out-of-plane
    deviator -(e11 + e22)/3, the shear as the mean of e12 and e21."""
    e11, e22 = eps[..., 0, 0], eps[..., 1, 1]
    t3 = (e11 + e22) / 3.0
    g = 0.5 * (eps[..., 0, 1] + eps[..., 1, 0])
    return np.sqrt((2.0 / 3.0) * ((e11 - t3) ** 2 + (e22 - t3) ** 2 + t3 ** 2 + 2.0 * g ** 2))


def _vm_eq_3d(eps):
    """Von Mises equivalent strain of a 3D field (elasticity.py:665-700)."""
    t3 = np.trace(eps, axis1=-2, axis2=-1) / 3.0
    dev = sum((eps[..., i, i] - t3) ** 2 for i in range(3))
    shear = sum((eps[..., i, j] + eps[..., j, i]) ** 2 for i, j in ((0, 1), (0, 2), (1, 2)))
    return np.sqrt((2.0 / 3.0) * (dev + 0.5 * shear))


def _e_nu(lam, mu):
    """(E, nu) of Lame moduli, guarded as the ramps' VTK output guards them."""
    return mu * (3.0 * lam + 2.0 * mu) / (lam + mu + 1e-30), lam / (2.0 * (lam + mu) + 1e-30)


def _rose_mu_sec_2d(eps, lam, mu, eta, floor_f, plane_mode):
    """The Rose secant shear modulus of a 2D field for the ramp's VTK output
    (linear_elastic_simulator.py:1766-1800): plane strain at e33 = 0; plane
    stress with e33 from five fixed-point steps of the isotropic relation
    e33 = -(3K - 2G)/(3K + 4G) (e11 + e22) from the linear guess, G taken
    before the last step."""
    exx, eyy, exy = eps[..., 0, 0], eps[..., 1, 1], eps[..., 0, 1]

    def g_of(ezz):
        t3 = (exx + eyy + ezz) / 3.0
        eq = np.sqrt((2.0 / 3.0) * ((exx - t3) ** 2 + (eyy - t3) ** 2 + (ezz - t3) ** 2 + 2.0 * exy ** 2))
        return np.maximum(mu * np.exp(-eta * eq), floor_f * mu)

    if plane_mode != "plane_stress":
        return g_of(0.0)
    K = lam + (2.0 / 3.0) * mu
    ezz = -lam / (lam + 2.0 * mu) * (exx + eyy)
    for _ in range(5):
        G = g_of(ezz)
        ezz = -(3.0 * K - 2.0 * G) / (3.0 * K + 4.0 * G) * (exx + eyy)
    return G


class _RampLog:
    """The ramps' per-step log (timestamp, elapsed time, step, driven strain
    and stress) and global log (every independent component), in the
    reference's column layout."""

    def __init__(self, dim, log_path, global_log_path, driving_component):
        import time as _time
        self.lbl = _COMP_LABELS.get(tuple(driving_component), "xx")
        self.ij = tuple(driving_component)
        self.comps = [(0, 0), (1, 1), (0, 1)] if dim == 2 else [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]
        self.f = open(log_path, "w", buffering=1) if log_path else None
        if self.f:
            hdr = (f"{'Timestamp':<20} {'Elapsed(s)':<12} {'Step':<8} {'Eps_' + self.lbl:<14} "
                   f"{'Sig_' + self.lbl + '(GPa)':<16}\n")
            self.f.write(hdr)
            self.f.write("-" * len(hdr.rstrip()) + "\n")
        self.g = open(global_log_path, "w", buffering=1) if global_log_path else None
        if self.g:
            ghdr = f"{'GlobalStep':<12} " + " ".join(f"{'Eps_' + _COMP_LABELS[c]:<14}" for c in self.comps) + " " + \
                   " ".join(f"{'Sig_' + _COMP_LABELS[c] + '(GPa)':<16}" for c in self.comps) + "\n"
            self.g.write(ghdr)
            self.g.write("-" * len(ghdr.rstrip()) + "\n")
        self.t0 = _time.time()

    def step(self, s, n_steps, epsM, sigM, console):
        import time as _time
        from datetime import datetime as _dt
        e, g = epsM[self.ij], sigM[self.ij]
        if console:
            print(f"step {s}/{n_steps}: eps_{self.lbl}={e:.4f}, sig_{self.lbl}={g / 1e9:.4f} GPa")
        if self.f:
            self.f.write(f"{_dt.now().strftime('%Y-%m-%d %H:%M:%S'):<20} {_time.time() - self.t0:<12.3f} {s:<8} "
                         f"{e:<14.6f} {g / 1e9:<16.6f}\n")
        if self.g:
            self.g.write(f"{s:<12} " + " ".join(f"{epsM[c]:<14.6f}" for c in self.comps) + " " +
                         " ".join(f"{sigM[c] / 1e9:<16.6f}" for c in self.comps) + "\n")

    def close(self, console):
        import time as _time
        from datetime import datetime as _dt
        total = _time.time() - self.t0
        m_, s_ = divmod(total, 60)
        h_, m_ = divmod(m_, 60)
        dur = (f"\nSimulation Finish Time: {_dt.now().strftime('%Y-%m-%d %H:%M:%S')}\nTotal Duration: {total:.2f} "
               f"seconds ({int(h_):d}h {int(m_):02d}m {int(s_):02d}s)\n")
        if self.f:
            self.f.write(dur)
            self.f.close()
        if self.g:
            self.g.close()
        if console:
            print(dur)


def _nl_ramp(dim, solve, lam, mu, mu_ref, target_strain_mask, target_values, n_steps, tol_macro, max_iter_macro,
             store, pixel, log_path, global_log_path, driving_component, enable_console, vtk_path, vtk_interval,
             solver_kw, vtk_moduli, secant_slopes=False):
    """Load ramp of the nonlinear drivers.  ``solve(eps_bar, eps_init)``
    returns (eps, sig, eps_mean, sig_mean) of one device solve; ``mu_ref`` is
    the shear modulus of the solver's reference medium (lambda is the mean
    lambda), whose isotropic compliance corrects the stress-controlled
    components; ``vtk_moduli(eps)`` gives the (E, nu) fields written with
    the VTK output.  Checkpoints carry the linear (E, nu) of (lambda, mu): the
    reference passes None there, which its writer cannot store."""
    chk_ival = solver_kw.pop("checkpoint_interval", None)
    chk_path = solver_kw.pop("checkpoint_path", "checkpoint")
    if chk_path and chk_ival not in (None, "none"):
        import os
        os.makedirs(os.path.dirname(chk_path) or ".", exist_ok=True)
    mask = np.asarray(target_strain_mask, dtype=bool)
    stress_mask = ~mask
    target_values = np.asarray(target_values, dtype=np.float64)
    lam_avg = float(np.mean(lam))
    E_ref = mu_ref * (3.0 * lam_avg + 2.0 * mu_ref) / (lam_avg + mu_ref)
    nu_ref = lam_avg / (2.0 * (lam_avg + mu_ref))
    log = _RampLog(dim, log_path, global_log_path, driving_component)
    cur = np.zeros((dim, dim))
    warm = None
    eps_macro_list, sig_macro_list, eps_list, sig_list = [], [], [], []
    for s in range(n_steps + 1):
        target_s = target_values * (s / n_steps)
        max_err = 0.0
        prev_e = prev_s = None  # secant history of the stress-controlled components, per load step
        for _ in range(max_iter_macro):
            cur[mask] = target_s[mask]
            eps, sig, epsM, sigM = solve(cur.copy(), warm)
            err = np.zeros((dim, dim))
            err[stress_mask] = target_s[stress_mask] - sigM[stress_mask]
            max_err = np.max(np.abs(err[stress_mask])) if np.any(stress_mask) else 0.0
            if max_err < tol_macro:
                break
            d = ((err - nu_ref * np.trace(err) * np.eye(dim)) / E_ref)[stress_mask]
            if secant_slopes:
                e_sc, s_sc = cur[stress_mask].copy(), np.asarray(sigM)[stress_mask].copy()
                if prev_e is not None:
                    de, ds = e_sc - prev_e, s_sc - prev_s
                    with np.errstate(divide="ignore", invalid="ignore"):
                        slope = ds / de
                    ok = np.isfinite(slope) & (np.abs(de) > 1e-14) & (slope > 0.01 * E_ref)
                    d[ok] = err[stress_mask][ok] / slope[ok]
                prev_e, prev_s = e_sc, s_sc
            cur[stress_mask] += d
        else:
            print(f"Warning: Macro loop did not converge at step {s} (err={max_err:.2e})")
        warm = eps
        eps_macro_list.append(epsM)
        sig_macro_list.append(sigM)
        if store:
            eps_list.append(eps)
            sig_list.append(sig)
        log.step(s, n_steps, epsM, sigM, enable_console)
        if chk_ival is not None and chk_ival not in ("none", "last"):
            name = None
            if chk_ival == "current":
                name = f"{chk_path}.h5"
            elif isinstance(chk_ival, int) and s % chk_ival == 0:
                name = f"{chk_path}_{s:06d}.h5"
            if name:
                _save_chk(dim, name, s, *_e_nu(lam, mu), eps, sig, epsM, sigM, pixel)
        if vtk_interval is not None and vtk_interval not in ("none", "last"):
            _vtk_step(vtk_interval, vtk_path, s, eps, sig, *vtk_moduli(eps), pixel)
    if chk_ival == "last":
        _save_chk(dim, f"{chk_path}_final.h5", n_steps, *_e_nu(lam, mu), eps, sig, epsM, sigM, pixel)
    if vtk_interval == "last" and vtk_path:
        from .vtk import export_to_vtk
        export_to_vtk(f"{vtk_path}_final.vtu", eps, sig, *vtk_moduli(eps), pixel, match_matplotlib_orientation=True)
    log.close(enable_console)
    return np.array(eps_macro_list), np.array(sig_macro_list), eps_list, sig_list


def _pop_landau_kw(solver_kw):
    """The Landau ramps' solver options (linear_elastic_simulator.py:2121-2127)."""
    return dict(solver=solver_kw.pop("solver", "dbfft"),
                strain_capping_enabled=solver_kw.pop("strain_capping_enabled", False),
                strain_capping_limit=solver_kw.pop("strain_capping_limit", None),
                strain_capping_tangent_ratio=solver_kw.pop("strain_capping_tangent_ratio", 0.1),
                strain_capping_type=solver_kw.pop("strain_capping_type", "piecewise"),
                strain_capping_smooth_power=solver_kw.pop("strain_capping_smooth_power", 1.0))


def secant_elastic_simulation_2d(lam, mu, d, k, target_strain_mask, target_values, n_steps=20, pixel=1.0, tol_ls=1e-6,
                                 max_iter_ls=400, tol_macro=1e-4, max_iter_macro=20, store=True,
                                 plane_mode="plane_strain", log_path=None, global_log_path=None,
                                 driving_component=(0, 0), enable_console=True, vtk_path=None, vtk_interval="none",
                                 **solver_kw):
    """Mixed stress/strain ramp with the secant-degradation law in 2D
    (linear_elastic_simulator.py:1353-1600); returns as
    linear_elastic_simulation_2d.  VTK moduli from the secant shear modulus
    of the final strain (:1567-1571)."""
    lam = np.asarray(lam, dtype=np.float64)
    mu = np.asarray(mu, dtype=np.float64)

    def solve(eb, init):
        return spectral_solver_secant_2d(lam, mu, d, k, eb, max_iter=max_iter_ls, tol=tol_ls, pixel=pixel,
                                         plane_mode=plane_mode, eps_init=init)

    def moduli(eps):
        return _e_nu(lam, mu * (1.0 - d * (1.0 - np.exp(-k * _vm_eq_2d(eps)))))

    return _nl_ramp(2, solve, lam, mu, float(mu.mean()), target_strain_mask, target_values, n_steps, tol_macro,
                    max_iter_macro, store, pixel, log_path, global_log_path, driving_component, enable_console,
                    vtk_path, vtk_interval, dict(solver_kw), moduli)


def rose_elastic_simulation_2d(lam, mu, eta, mu_floor_fraction=0.1, target_strain_mask=None, target_values=None,
                               n_steps=20, pixel=1.0, tol_ls=1e-6, max_iter_ls=400, tol_macro=1e-4, max_iter_macro=20,
                               store=True, plane_mode="plane_strain", log_path=None, global_log_path=None,
                               driving_component=(0, 0), enable_console=True, vtk_path=None, vtk_interval="none",
                               **solver_kw):
    """Mixed stress/strain ramp with the Rose law in 2D
    (linear_elastic_simulator.py:1603-1856): the compliance of the solver's
    reference medium (mean lambda, (1 + floor) mean mu / 2) corrects the
    stress-controlled components (:1640-1652); returns as
    linear_elastic_simulation_2d."""
    lam = np.asarray(lam, dtype=np.float64)
    mu = np.asarray(mu, dtype=np.float64)

    def solve(eb, init):
        return spectral_solver_rose_2d(lam, mu, eta, mu_floor_fraction, eps_bar=eb, max_iter=max_iter_ls, tol=tol_ls,
                                       pixel=pixel, plane_mode=plane_mode, eps_init=init)

    def moduli(eps):
        return _e_nu(lam, _rose_mu_sec_2d(eps, lam, mu, eta, mu_floor_fraction, plane_mode))

    mu_ref = 0.5 * (1.0 + mu_floor_fraction) * float(mu.mean())
    return _nl_ramp(2, solve, lam, mu, mu_ref, target_strain_mask, target_values, n_steps, tol_macro, max_iter_macro,
                    store, pixel, log_path, global_log_path, driving_component, enable_console, vtk_path,
                    vtk_interval, dict(solver_kw), moduli)


def secant_elastic_simulation_3d(lam, mu, d, k, target_strain_mask, target_values, n_steps=20, pixel=1.0, tol_ls=1e-6,
                                 max_iter_ls=400, tol_macro=1e-4, max_iter_macro=20, store=True, log_path=None,
                                 global_log_path=None, driving_component=(0, 0), enable_console=True, vtk_path=None,
                                 vtk_interval="none", **solver_kw):
    """Mixed stress/strain ramp with the secant-degradation law in 3D
    (linear_elastic_simulator.py:1857-2054); returns as
    linear_elastic_simulation_3d."""
    lam = np.asarray(lam, dtype=np.float64)
    mu = np.asarray(mu, dtype=np.float64)

    def solve(eb, init):
        return spectral_solver_secant_3d(lam, mu, d, k, eb, max_iter=max_iter_ls, tol=tol_ls, pixel=pixel,
                                         eps_init=init)

    def moduli(eps):
        return _e_nu(lam, mu * (1.0 - d * (1.0 - np.exp(-k * _vm_eq_3d(eps)))))

    return _nl_ramp(3, solve, lam, mu, float(mu.mean()), target_strain_mask, target_values, n_steps, tol_macro,
                    max_iter_macro, store, pixel, log_path, global_log_path, driving_component, enable_console,
                    vtk_path, vtk_interval, dict(solver_kw), moduli)


def landau_elastic_simulation_2d(lam, mu, v1, v2, v3, g1, g2, g3, g4, target_strain_mask, target_values, n_steps=20,
                                 pixel=1.0, tol_ls=1e-6, max_iter_ls=400, tol_macro=1e-4, max_iter_macro=20,
                                 store=True, plane_mode="plane_strain", log_path=None, global_log_path=None,
                                 driving_component=(0, 0), enable_console=True, vtk_path=None, vtk_interval="none",
                                 **solver_kw):
    """Mixed stress/strain ramp with the Landau law in 2D
    (linear_elastic_simulator.py:2055-2284): the stress-controlled
    components take the secant slope of the last two macro iterates where it
    is finite and above 1 % of the reference Young's modulus (:2186-2204),
    else the compliance step; plane stress passes one e33 state through
    every solve (:2146).  Solver options (``solver``, strain capping) come in
    ``solver_kw``; returns as linear_elastic_simulation_2d."""
    lam = np.asarray(lam, dtype=np.float64)
    mu = np.asarray(mu, dtype=np.float64)
    skw = dict(solver_kw)
    lkw = _pop_landau_kw(skw)
    e33_state = {} if plane_mode == "plane_stress" else None

    def solve(eb, init):
        return spectral_solver_landau_2d(lam, mu, v1, v2, v3, g1, g2, g3, g4, eb, max_iter=max_iter_ls, tol=tol_ls,
                                         pixel=pixel, plane_mode=plane_mode, eps_init=init, e33_state=e33_state,
                                         **lkw)

    return _nl_ramp(2, solve, lam, mu, float(mu.mean()), target_strain_mask, target_values, n_steps, tol_macro,
                    max_iter_macro, store, pixel, log_path, global_log_path, driving_component, enable_console,
                    vtk_path, vtk_interval, skw, lambda eps: _e_nu(lam, mu), secant_slopes=True)


def landau_elastic_simulation_3d(lam, mu, v1, v2, v3, g1, g2, g3, g4, target_strain_mask, target_values, n_steps=20,
                                 pixel=1.0, tol_ls=1e-6, max_iter_ls=400, tol_macro=1e-4, max_iter_macro=20,
                                 store=True, log_path=None, global_log_path=None, driving_component=(0, 0),
                                 enable_console=True, vtk_path=None, vtk_interval="none", **solver_kw):
    """Mixed stress/strain ramp with the Landau law in 3D
    (linear_elastic_simulator.py:2287-2517), the 2D ramp's macro loop with
    3x3 tensors.  The global log carries all six independent components
    under the reference's six-column header (the reference writes xx, yy and
    xz there only, :2463-2467)."""
    lam = np.asarray(lam, dtype=np.float64)
    mu = np.asarray(mu, dtype=np.float64)
    skw = dict(solver_kw)
    lkw = _pop_landau_kw(skw)

    def solve(eb, init):
        return spectral_solver_landau_3d(lam, mu, v1, v2, v3, g1, g2, g3, g4, eb, max_iter=max_iter_ls, tol=tol_ls,
                                         pixel=pixel, eps_init=init, **lkw)

    return _nl_ramp(3, solve, lam, mu, float(mu.mean()), target_strain_mask, target_values, n_steps, tol_macro,
                    max_iter_macro, store, pixel, log_path, global_log_path, driving_component, enable_console,
                    vtk_path, vtk_interval, skw, lambda eps: _e_nu(lam, mu), secant_slopes=True)
