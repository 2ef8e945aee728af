"""Drop-in 3D finite-strain Newton-Krylov step backed by the CUDA library.

``finite_strain_solver_step_3d`` keeps the signature and return value of
mgkmc/finite_strain_simulator.py:2967-3168 for ``solver="newton_cg"``
(numpy tensor-first arrays in and out).  ``Ghat4``, ``I2``, ``I4``, ``I4rt``
are accepted and ignored: the projection and the identities are applied on
the fly, and only lambda = C4[0,0,1,1] and mu = C4[0,1,0,1] are read from
``C4``.  The 81-component tangent is never formed, so ``K4`` is returned as
None (no in-scope caller uses it: aqs.py:289 discards it).  ``Fs3dSolver``
is the device-resident interface (torch CUDA tensors, plan reused across load
steps); ``simulate_3d`` runs the incremental load ramp of
finite_strain_simulation_3d (:3175-3298) with an eigen-deformation field.
"""
import ctypes

import numpy as np

from . import _lib as L

_MODEL = {"svk": 0, "neo_hookean": 1}


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("mgkmc_b200 needs a CUDA device (no CPU fallback)")
    return torch


def build_finite_strain_bc_3d(driving_component, eps_target_step, mixed_targets, ndim=3, F_bar_initial=None):
    """mgkmc/finite_strain_simulator.py:2852-2899 (host-side bookkeeping)."""
    F_bar = np.eye(ndim) if F_bar_initial is None else F_bar_initial.copy()
    F_mask = np.zeros((ndim, ndim), dtype=bool)
    P_target = np.zeros((ndim, ndim))
    P_mask = np.zeros((ndim, ndim), dtype=bool)
    i_d, j_d = driving_component
    F_bar[i_d, j_d] = 1.0 + eps_target_step if i_d == j_d else eps_target_step
    F_mask[i_d, j_d] = True
    for a in range(ndim):
        for b in range(ndim):
            if a != b and (a, b) != (i_d, j_d):
                F_bar[a, b] = 0.0
                F_mask[a, b] = True
    for k in range(ndim):
        if k == i_d and i_d == j_d:
            continue
        if (k, k) in mixed_targets:
            P_target[k, k] = mixed_targets[(k, k)]
            P_mask[k, k] = True
        else:
            F_bar[k, k] = 1.0
            F_mask[k, k] = True
    return F_bar, F_mask, P_target, P_mask


class Fs3dSolver:
    """Plan-owning 3D finite-strain solver on one device.  ``precision``:
    "fp64" (the reference's arithmetic) or "mixed" (FP32 Krylov matvecs; the
    Newton residual, CG vectors, inner products and norms stay FP64)."""

    def __init__(self, nx, ny, nz, model="svk", device=None, precision="fp64"):
        torch = _torch()
        self.shape = (int(nx), int(ny), int(nz))
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            L.check(L.lib().mgk_fs3d_create(*self.shape, _MODEL[model], ctypes.byref(h)), "mgk_fs3d_create")
        self._h = h
        self.precision = precision
        if precision != "fp64":
            L.check(L.lib().mgk_fs3d_set_precision(h, L.MIXED), "mgk_fs3d_set_precision")
        self._keep = {}
        self.info = L.FsInfo()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                L.lib().mgk_fs3d_destroy(h)
            except Exception:
                pass
            self._h = None

    def set_material(self, lam, mu, Fp=None, stream=None):
        self._keep["m"] = (lam, mu, Fp)
        L.check(L.lib().mgk_fs3d_set_material(self._h, L.ptr(lam), L.ptr(mu), L.ptr(Fp), L.stream_ptr(stream)),
                "mgk_fs3d_set_material")

    def set_F(self, F, stream=None):
        L.check(L.lib().mgk_fs3d_set_F(self._h, L.ptr(F), L.stream_ptr(stream)), "mgk_fs3d_set_F")

    def step(self, F_bar, driving_component=(0, 0), P_target=None, P_mask=None, E_avg=100e9, nu_avg=0.3,
             tol_NW=1e-5, tol_CG=1e-6, max_NW=50, tol_macro=1e6, max_iter_macro=20, stream=None):
        D9 = ctypes.c_double * 9
        fb = D9(*np.asarray(F_bar, dtype=np.float64).ravel())
        pt = None if P_target is None else D9(*np.asarray(P_target, dtype=np.float64).ravel())
        pm = None if P_mask is None else (ctypes.c_int * 9)(*[int(v) for v in np.asarray(P_mask).ravel()])
        out = D9()
        st = L.lib().mgk_fs3d_step(self._h, fb, int(driving_component[0]), int(driving_component[1]), pt, pm,
                                   float(E_avg), float(nu_avg), float(tol_NW), float(tol_CG), int(max_NW),
                                   float(tol_macro), int(max_iter_macro), out, ctypes.byref(self.info),
                                   L.stream_ptr(stream))
        if st == L.NOT_CONVERGED:
            raise ValueError(L.lib().mgk_last_error().decode())
        L.check(st, "mgk_fs3d_step")
        return np.array(out[:]).reshape(3, 3), self.info

    def profile_kernels(self, fp32=False, reps=20, stream=None):
        """Mean ms of the six kernels of one Krylov iteration (z fwd, y, x+G,
        y inv, z inv, update); leaves the Krylov vectors unspecified."""
        ms = (ctypes.c_float * 6)()
        L.check(L.lib().mgk_fs3d_profile(self._h, 1 if fp32 else 0, int(reps), ms, L.stream_ptr(stream)),
                "mgk_fs3d_profile")
        return list(ms)

    def autotune(self, reps=5, stream=None):
        """Keeps the faster kernel family (1 warp-line, 0 CTA-wide) for this
        plan, timed on its current state (call after a step)."""
        ch, ms = ctypes.c_int(), ctypes.c_float()
        L.check(L.lib().mgk_fs3d_autotune(self._h, int(reps), ctypes.byref(ch), ctypes.byref(ms),
                                          L.stream_ptr(stream)), "mgk_fs3d_autotune")
        return ch.value, ms.value

    def get(self, F_out=None, P_out=None, sig_out=None, stream=None):
        L.check(L.lib().mgk_fs3d_get(self._h, L.ptr(F_out), L.ptr(P_out), L.ptr(sig_out), L.stream_ptr(stream)),
                "mgk_fs3d_get")


_PLANS = {}


def finite_strain_solver_step_3d(F, F_bar, Ghat4=None, C4=None, I2=None, I4=None, I4rt=None, Fp=None,
                                 driving_component=(0, 0), P_target=None, P_mask=None, E_avg=100e9, nu_avg=0.3,
                                 tol_NW=1e-5, tol_CG=1e-6, max_NW=50, tol_macro=1e6, max_iter_macro=20,
                                 enable_console=True, model_type="svk", A_m=0.0, B_m=0.0, C_m=0.0, solver="al",
                                 pixel=1.0, lam=None, mu=None, **unused):
    """One mixed-BC load step (mgkmc/finite_strain_simulator.py:2967-3168),
    Newton-Krylov path.  Returns (F, P, Sig, None, F_bar_current)."""
    if solver not in ("newton_cg", "newton"):
        raise NotImplementedError(f"solver={solver!r}: only the Newton-Krylov path runs on the GPU")
    if model_type not in _MODEL:
        raise NotImplementedError(f"model_type={model_type!r}: SVK and Neo-Hookean run on the GPU")
    torch = _torch()
    F = np.ascontiguousarray(F, dtype=np.float64)
    shape = F.shape[2:]
    if lam is None or mu is None:
        lam = np.ascontiguousarray(C4[0, 0, 1, 1])
        mu = np.ascontiguousarray(C4[0, 1, 0, 1])
    dev = torch.device("cuda", torch.cuda.current_device())
    key = (shape, model_type, dev.index)
    s = _PLANS.get(key)
    if s is None:
        s = _PLANS[key] = Fs3dSolver(*shape, model=model_type)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(dev)
    s.set_material(t(lam), t(mu), None if Fp is None else t(Fp))
    s.set_F(t(F))
    Fb, info = s.step(F_bar, driving_component, P_target, P_mask, E_avg, nu_avg, tol_NW, tol_CG, max_NW, tol_macro,
                      max_iter_macro)
    Fo = torch.empty((3, 3) + tuple(shape), dtype=torch.float64, device=dev)
    Po = torch.empty_like(Fo)
    So = torch.empty_like(Fo)
    s.get(Fo, Po, So)
    if enable_console:
        print(f"finite strain step: {info.macro_iterations} macro, {info.newton_iterations} Newton, "
              f"{info.krylov_iterations} CG iterations")
    return Fo.cpu().numpy(), Po.cpu().numpy(), So.cpu().numpy(), None, Fb


def simulate_3d(E, nu, Fp, eps_target, n_steps, driving_component=(0, 0), mixed_targets=None, model="neo_hookean",
                tol_NW=1e-8, tol_CG=1e-6, max_NW=50, tol_macro=1e6, max_iter_macro=20, solver=None, precision="fp64"):
    """Incremental load ramp of finite_strain_simulation_3d (:3270-3298) with
    an eigen-deformation field F_p (that driver passes Fp=None, :3282).
    Returns the list of (F_bar, info) per step; the solver keeps the field."""
    torch = _torch()
    mixed_targets = {} if mixed_targets is None else mixed_targets
    shape = E.shape
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    dev = torch.device("cuda", torch.cuda.current_device())
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(dev)
    s = solver if solver is not None else Fs3dSolver(*shape, model=model, precision=precision)
    s.set_material(t(lam), t(mu), None if Fp is None else t(Fp))
    s.set_F(t(np.einsum("ij,xyz->ijxyz", np.eye(3), np.ones(shape))))
    F_bar_init = None
    out = []
    for eps in np.linspace(0.0, eps_target, n_steps + 1):
        F_bar, _, P_tgt, P_mask = build_finite_strain_bc_3d(driving_component, eps, mixed_targets,
                                                            F_bar_initial=F_bar_init)
        Fb, info = s.step(F_bar, driving_component, P_tgt, P_mask, float(E.mean()), float(nu.mean()), tol_NW, tol_CG,
                          max_NW, tol_macro, max_iter_macro)
        F_bar_init = Fb
        out.append((Fb, dict(newton=info.newton_iterations, krylov=info.krylov_iterations,
                             macro=info.macro_iterations, sig_mean=np.array(info.sig_mean).reshape(3, 3))))
    return s, out
