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
from .linear_elastic_simulator import _vtk_final, _vtk_step

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


_COMP = {(0, 0): "xx", (1, 1): "yy", (2, 2): "zz", (0, 1): "xy", (0, 2): "xz", (1, 2): "yz", (1, 0): "yx",
         (2, 0): "zx", (2, 1): "zy"}


def finite_strain_simulation_3d(E, nu, driving_component, eps_target, n_steps, mixed_targets=None, pixel=1.0,
                                tol_NW=1e-5, tol_CG=1e-6, max_NW=20, tol_macro=1e6, max_iter_macro=20, store=True,
                                log_path=None, global_log_path=None, enable_console=True,
                                checkpoint_interval="none", checkpoint_path=None, vtk_interval="none", vtk_path=None,
                                model_type="svk", A_m=0.0, B_m=0.0, C_m=0.0, solver="al", Fp=None, precision="fp64",
                                **unused):
    """Incremental 3D finite-strain load ramp (finite_strain_simulator.py:3175-3414)
    on one device-resident plan: per load step s the boundary conditions of
    build_finite_strain_bc_3d at eps_target * s / n_steps (seeded with the
    previous step's F_bar), one Newton-Krylov load step from the previous
    field.  Returns (F_macro, Sig_macro, P_macro, F list, Sig list) like the
    reference.  ``Fp`` (tensor-first, optional) is an eigen-deformation field
    the reference's driver does not take (it passes Fp=None, :3282); None
    reproduces the reference.  Only solver="newton_cg" runs here."""
    import time as _time
    from datetime import datetime as _dt
    if solver not in ("newton_cg", "newton"):
        raise NotImplementedError(f"solver={solver!r}: only the Newton-Krylov path runs on the GPU")
    if model_type not in _MODEL:
        raise NotImplementedError(f"model_type={model_type!r}: SVK and Neo-Hookean run on the GPU")
    torch = _torch()
    mixed_targets = {} if mixed_targets is None else mixed_targets
    E = np.ascontiguousarray(E, dtype=np.float64)
    nu = np.ascontiguousarray(nu, dtype=np.float64)
    shape = E.shape
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    dev = torch.device("cuda", torch.cuda.current_device())
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(dev)
    s_ = Fs3dSolver(*shape, model=model_type, precision=precision)
    s_.set_material(t(lam), t(mu), None if Fp is None else t(Fp))
    F = torch.zeros((3, 3) + shape, dtype=torch.float64, device=dev)
    for i in range(3):
        F[i, i] = 1.0
    s_.set_F(F)
    P = torch.empty_like(F)
    Sig = torch.empty_like(F)
    lbl = _COMP.get(tuple(driving_component), "xx")
    log_f = open(log_path, "w", buffering=1) if log_path else None
    if log_f:
        hdr = (f"{'Timestamp':<20} {'Elapsed(s)':<12} {'Step':<8} {'F_' + lbl:<14} {'Eng_strain_' + lbl:<20} "
               f"{'Sig_' + lbl + '(GPa)':<18}\n")
        log_f.write(hdr)
        log_f.write("-" * len(hdr.rstrip()) + "\n")
    glog_f = open(global_log_path, "w", buffering=1) if global_log_path else None
    six = [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]
    if glog_f:
        ghdr = (f"{'Step':<8} " + " ".join(f"{'F_' + _COMP[c]:<12}" for c in six) + " " +
                " ".join(f"{'EngStr_' + _COMP[c]:<14}" for c in six[:3]) + " " +
                " ".join(f"{'P_' + _COMP[c] + '(GPa)':<14}" for c in six) + " " +
                " ".join(f"{'Sig_' + _COMP[c] + '(GPa)':<16}" for c in six) + "\n")
        glog_f.write(ghdr)
        glog_f.write("-" * len(ghdr.rstrip()) + "\n")
    t0 = _time.time()
    F_macro, Sig_macro, P_macro, F_list, Sig_list = [], [], [], [], []
    F_bar_init = None
    E_avg, nu_avg = float(E.mean()), float(nu.mean())
    for s, eps_s in enumerate(np.linspace(0.0, eps_target, n_steps + 1)):
        F_bar, _, P_tgt, P_mask = build_finite_strain_bc_3d(driving_component, eps_s, mixed_targets,
                                                            F_bar_initial=F_bar_init)
        F_bar_init, info = s_.step(F_bar, driving_component, P_tgt, P_mask, E_avg, nu_avg, tol_NW, tol_CG, max_NW,
                                   tol_macro, max_iter_macro)
        if enable_console:
            print(f"finite strain step: {info.macro_iterations} macro, {info.newton_iterations} Newton, "
                  f"{info.krylov_iterations} CG iterations")
        s_.get(F, P, Sig)
        F_mac = F.mean(dim=(2, 3, 4)).cpu().numpy()
        P_mac = P.mean(dim=(2, 3, 4)).cpu().numpy()
        S_mac = Sig.mean(dim=(2, 3, 4)).cpu().numpy()
        F_macro.append(F_mac)
        Sig_macro.append(S_mac)
        P_macro.append(P_mac)
        if store:
            F_list.append(F.cpu().numpy())
            Sig_list.append(Sig.cpu().numpy())
        i, j = driving_component
        F_drv = F_mac[i, j]
        eng = F_drv - (1.0 if i == j else 0.0)
        if enable_console:
            print(f"step {s}/{n_steps}: F_{lbl}={F_drv:.5f}, eng_strain={eng:.5f}, Sig_{lbl}={S_mac[i, j] / 1e9:.4f} GPa")
        if log_f:
            log_f.write(f"{_dt.now().strftime('%Y-%m-%d %H:%M:%S'):<20} {_time.time() - t0:<12.3f} {s:<8} "
                        f"{F_drv:<14.6f} {eng:<20.6f} {S_mac[i, j] / 1e9:<18.6f}\n")
        if glog_f:
            glog_f.write(f"{s:<8} " + " ".join(f"{F_mac[c]:<12.6f}" for c in six) + " " +
                         " ".join(f"{F_mac[c] - 1:<14.6f}" for c in six[:3]) + " " +
                         " ".join(f"{P_mac[c] / 1e9:<14.6f}" for c in six) + " " +
                         " ".join(f"{S_mac[c] / 1e9:<16.6f}" for c in six) + "\n")
        if checkpoint_path is not None and checkpoint_interval not in (None, "none", "last"):
            name = None
            if checkpoint_interval == "current":
                name = checkpoint_path
            elif isinstance(checkpoint_interval, int) and s % checkpoint_interval == 0:
                name = f"{checkpoint_path}_{s:06d}"
            if name:
                _checkpoint(name, s, E, nu, F, Sig, F_mac, S_mac, pixel)
        if vtk_path is not None:
            _vtk_step(vtk_interval, vtk_path, s, *_vtk_fields_3d(F, Sig), E, nu, pixel)
    if checkpoint_path is not None and (checkpoint_interval == "last" or (
            isinstance(checkpoint_interval, int) and n_steps % checkpoint_interval != 0)):
        _checkpoint(f"{checkpoint_path}_final", n_steps, E, nu, F, Sig, F_macro[-1], Sig_macro[-1], pixel)
    if vtk_path is not None:
        _vtk_final(vtk_interval, vtk_path, n_steps, *_vtk_fields_3d(F, Sig), E, nu, pixel)
    total = _time.time() - t0
    m_, sec = divmod(total, 60)
    h_, m_ = divmod(m_, 60)
    if log_f:
        log_f.write(f"\nSimulation Finish Time: {_dt.now().strftime('%Y-%m-%d %H:%M:%S')}\nTotal Duration: "
                    f"{total:.2f} seconds ({int(h_):d}h {int(m_):02d}m {int(sec):02d}s)\n")
        log_f.close()
    if glog_f:
        glog_f.close()
    return np.array(F_macro), np.array(Sig_macro), np.array(P_macro), F_list, Sig_list


def _vtk_fields_3d(F, Sig):
    """The fields the reference's ramp writes to VTK (:3367-3370): the
    Green-Lagrange strain and the Cauchy stress, spatial-first numpy."""
    torch = _torch()
    E_GL = 0.5 * (torch.einsum("kixyz,kjxyz->ijxyz", F, F) - torch.eye(3, dtype=F.dtype, device=F.device)
                  .reshape(3, 3, 1, 1, 1))
    return E_GL.permute(2, 3, 4, 0, 1).cpu().numpy(), Sig.permute(2, 3, 4, 0, 1).cpu().numpy()


def _checkpoint(path, step, E, nu, F, Sig, F_mac, S_mac, pixel):
    """The reference's checkpoint of a finite-strain step (:3351-3356): the
    Green-Lagrange strain and the Cauchy stress, spatial-first."""
    from . import checkpoint as C
    torch = _torch()
    E_GL = 0.5 * (torch.einsum("kixyz,kjxyz->ijxyz", F, F) - torch.eye(3, dtype=F.dtype, device=F.device)
                  .reshape(3, 3, 1, 1, 1))
    C.save_checkpoint_3d(path, step, E, nu, E_GL.permute(2, 3, 4, 0, 1).cpu().numpy(),
                         Sig.permute(2, 3, 4, 0, 1).cpu().numpy(), F_mac, S_mac, pixel)


# ------------------------------------- 2D plane strain and plane stress ---
_PLANE = (0, 2)  # 2D tensor index -> index in the embedded (nx, 1, ny) plan


def _embed_2d(A2, fill, torch, dev):
    """(2,2,nx,ny) -> tensor-first (3,3,nx,1,ny) device tensor; the out-of-plane
    diagonal entry is ``fill``."""
    A2 = torch.as_tensor(np.ascontiguousarray(A2, dtype=np.float64) if not hasattr(A2, "data_ptr") else A2,
                         dtype=torch.float64, device=dev)
    nx, ny = A2.shape[2:]
    A3 = torch.zeros((3, 3, nx, 1, ny), dtype=torch.float64, device=dev)
    for a, i in enumerate(_PLANE):
        for b, j in enumerate(_PLANE):
            A3[i, j, :, 0, :] = A2[a, b]
    A3[1, 1] = fill
    return A3


def _extract_2d(A3):
    return np.stack([np.stack([A3[i, j, :, 0, :] for j in _PLANE]) for i in _PLANE])


def _embed_small(M2, fill, dtype=np.float64):
    M3 = np.zeros((3, 3), dtype=dtype)
    for a, i in enumerate(_PLANE):
        for b, j in enumerate(_PLANE):
            M3[i, j] = M2[a][b]
    M3[1, 1] = fill
    return M3


class Fs2dSolver:
    """2D finite-strain solver: the 3D plan of an (nx, 1, ny) grid with the
    out-of-plane axis y (F_yy = 1) and the 2D Newton norm.  plane_mode
    "plane_strain" (``mgk_fs3d_set_plane_strain``) or "plane_stress"
    (``mgk_fs3d_set_plane_stress``: the material's lam is the plane-stress
    lambda E nu / (1 - nu^2); the laws are the reference's plane-stress ones,
    the Neo-Hookean with its per-voxel out-of-plane Newton solve, and the
    Cauchy stress carries the out-of-plane stretch F33).  Fields in and out
    are the reference's tensor-first (2, 2, nx, ny)."""

    def __init__(self, nx, ny, model="svk", precision="fp64", device=None, plane_mode="plane_strain"):
        if plane_mode not in ("plane_strain", "plane_stress"):
            raise ValueError(f"plane_mode={plane_mode!r}")
        self.nx, self.ny = int(nx), int(ny)
        self.plane_mode = plane_mode
        self.s = Fs3dSolver(self.nx, 1, self.ny, model=model, precision=precision, device=device)
        if plane_mode == "plane_stress":
            L.check(L.lib().mgk_fs3d_set_plane_stress(self.s._h, 1), "mgk_fs3d_set_plane_stress")
        else:
            L.check(L.lib().mgk_fs3d_set_plane_strain(self.s._h, 1), "mgk_fs3d_set_plane_strain")
        self.device = self.s.device

    def set_material(self, lam, mu, Fp=None, stream=None):
        torch = _torch()
        t = lambda a: torch.as_tensor(a, dtype=torch.float64, device=self.device).reshape(self.nx, 1, self.ny)
        self._keep = (t(lam).contiguous(), t(mu).contiguous(),
                      None if Fp is None else _embed_2d(Fp, 1.0, torch, self.device))
        self.s.set_material(*self._keep, stream=stream)

    def set_F(self, F, stream=None):
        torch = _torch()
        self._F = _embed_2d(F, 1.0, torch, self.device)
        self.s.set_F(self._F, stream=stream)

    def step(self, F_bar, driving_component=(0, 0), P_target=None, P_mask=None, E_avg=100e9, nu_avg=0.3,
             tol_NW=1e-5, tol_CG=1e-6, max_NW=50, tol_macro=1e6, max_iter_macro=20, stream=None):
        i, j = driving_component
        Fb3, info = self.s.step(_embed_small(F_bar, 1.0), (_PLANE[i], _PLANE[j]),
                                None if P_target is None else _embed_small(P_target, 0.0),
                                None if P_mask is None else _embed_small(P_mask, False, bool), E_avg, nu_avg, tol_NW,
                                tol_CG, max_NW, tol_macro, max_iter_macro, stream=stream)
        return Fb3[np.ix_(_PLANE, _PLANE)].copy(), info

    def get(self, stream=None):
        """(F, P, Cauchy stress) as numpy (2, 2, nx, ny)."""
        torch = _torch()
        F3 = torch.empty((3, 3, self.nx, 1, self.ny), dtype=torch.float64, device=self.device)
        P3, S3 = torch.empty_like(F3), torch.empty_like(F3)
        self.s.get(F3, P3, S3, stream=stream)
        return tuple(_extract_2d(t.cpu().numpy()) for t in (F3, P3, S3))


_PLANS2 = {}


def finite_strain_solver_step_2d(F, F_bar, Ghat4=None, C4=None, I2=None, I4=None, I4rt=None, Fp=None,
                                 driving_component=(0, 0), P_target=None, P_mask=None, E_avg=100e9, nu_avg=0.3,
                                 tol_NW=1e-5, tol_CG=1e-6, max_NW=50, tol_macro=1e6, max_iter_macro=20,
                                 enable_console=True, model_type="svk", plane_mode="plane_strain", A_m=0.0, B_m=0.0,
                                 C_m=0.0, solver="al", pixel=1.0, lam=None, mu=None, **unused):
    """One mixed-BC 2D load step (mgkmc/finite_strain_simulator.py:2356-2572),
    Newton-Krylov path, plane strain or plane stress (SVK, Neo-Hookean):
    returns (F, P, Sig, None, F_bar_current) with (2, 2, nx, ny) fields.  The
    Lame fields come from ``C4`` (C4[0,0,1,1] and C4[0,1,0,1], the reference's
    build_C4_2d, whose lambda is the plane-stress one in plane stress) or
    ``lam``/``mu``."""
    if solver not in ("newton_cg", "newton"):
        raise NotImplementedError(f"solver={solver!r}: only the Newton-Krylov path runs on the GPU")
    if model_type not in _MODEL:
        raise NotImplementedError(f"model_type={model_type!r}: SVK and Neo-Hookean run on the GPU")
    if plane_mode not in ("plane_strain", "plane_stress"):
        raise ValueError(f"plane_mode={plane_mode!r}")
    torch = _torch()
    F = np.ascontiguousarray(F, dtype=np.float64)
    nx, ny = F.shape[2:]
    if lam is None or mu is None:
        lam = np.ascontiguousarray(C4[0, 0, 1, 1])
        mu = np.ascontiguousarray(C4[0, 1, 0, 1])
    dev = torch.device("cuda", torch.cuda.current_device())
    key = (nx, ny, model_type, plane_mode, dev.index)
    s = _PLANS2.get(key)
    if s is None:
        s = _PLANS2[key] = Fs2dSolver(nx, ny, model=model_type, plane_mode=plane_mode)
    s.set_material(lam, mu, Fp)
    s.set_F(F)
    Fb, info = s.step(F_bar, driving_component, P_target, P_mask, E_avg, nu_avg, tol_NW, tol_CG, max_NW, tol_macro,
                      max_iter_macro)
    Fo, Po, So = s.get()
    if enable_console:
        print(f"finite strain 2D step: {info.macro_iterations} macro, {info.newton_iterations} Newton, "
              f"{info.krylov_iterations} CG iterations")
    return Fo, Po, So, None, Fb


def build_finite_strain_bc(driving_component, eps_target_step, mixed_targets, plane_mode="plane_strain", ndim=2,
                           F_bar_initial=None):
    """2D boundary conditions of a load step (finite_strain_simulator.py:1912-1979):
    the same rule as build_finite_strain_bc_3d with ndim = 2 (``plane_mode``
    does not change it)."""
    return build_finite_strain_bc_3d(driving_component, eps_target_step, mixed_targets, ndim=ndim,
                                     F_bar_initial=F_bar_initial)


def finite_strain_simulation_2d(E, nu, driving_component, eps_target, n_steps, mixed_targets=None,
                                plane_mode="plane_strain", pixel=1.0, tol_NW=1e-5, tol_CG=1e-6, max_NW=20,
                                tol_macro=1e6, max_iter_macro=20, store=True, log_path=None, global_log_path=None,
                                enable_console=True, checkpoint_interval="none", checkpoint_path=None,
                                vtk_interval="none", vtk_path=None, model_type="svk", A_m=0.0, B_m=0.0, C_m=0.0,
                                solver="al", Fp=None, precision="fp64", **unused):
    """Incremental 2D finite-strain ramp (finite_strain_simulator.py:2580-2851),
    plane strain or plane stress with the plane-stress lambda
    E nu / (1 - nu^2) of build_C4_2d, on one device-resident embedded plan
    (``Fs2dSolver``): per load step the boundary conditions of
    build_finite_strain_bc at eps_target * s / n_steps (seeded with the
    previous F_bar), one Newton-Krylov load step from the previous field.
    Returns (F_macro, Sig_macro, P_macro, F list, Sig list) with (2, 2, nx, ny)
    fields.  ``Fp`` is an optional eigen-deformation field (the reference's
    driver passes none)."""
    import time as _time
    from datetime import datetime as _dt
    if solver not in ("newton_cg", "newton"):
        raise NotImplementedError(f"solver={solver!r}: only the Newton-Krylov path runs on the GPU")
    mixed_targets = {} if mixed_targets is None else mixed_targets
    E = np.ascontiguousarray(E, dtype=np.float64)
    nu = np.ascontiguousarray(nu, dtype=np.float64)
    nx, ny = E.shape
    if plane_mode == "plane_stress":
        lam = E * nu / (1.0 - nu ** 2)
    else:
        lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    s_ = Fs2dSolver(nx, ny, model=model_type, precision=precision, plane_mode=plane_mode)
    s_.set_material(lam, mu, Fp)
    s_.set_F(np.einsum("ij,xy->ijxy", np.eye(2), np.ones((nx, ny))))
    lbl = _COMP.get(tuple(driving_component), "xx")
    log_f = open(log_path, "w", buffering=1) if log_path else None
    if log_f:
        hdr = (f"{'Timestamp':<20} {'Elapsed(s)':<12} {'Step':<8} {'F_' + lbl:<14} {'Eng_strain_' + lbl:<20} "
               f"{'Sig_' + lbl + '(GPa)':<18}\n")
        log_f.write(hdr)
        log_f.write("-" * len(hdr.rstrip()) + "\n")
    glog_f = open(global_log_path, "w", buffering=1) if global_log_path else None
    t0 = _time.time()
    F_macro, Sig_macro, P_macro, F_list, Sig_list = [], [], [], [], []
    F_bar_init = None
    E_avg, nu_avg = float(E.mean()), float(nu.mean())
    for s, eps_s in enumerate(np.linspace(0.0, eps_target, n_steps + 1)):
        F_bar, _, P_tgt, P_mask = build_finite_strain_bc(driving_component, eps_s, mixed_targets, plane_mode,
                                                         F_bar_initial=F_bar_init)
        F_bar_init, info = s_.step(F_bar, driving_component, P_tgt, P_mask, E_avg, nu_avg, tol_NW, tol_CG, max_NW,
                                   tol_macro, max_iter_macro)
        F, P, Sig = s_.get()
        F_mac, P_mac, S_mac = F.mean(axis=(2, 3)), P.mean(axis=(2, 3)), Sig.mean(axis=(2, 3))
        F_macro.append(F_mac)
        P_macro.append(P_mac)
        Sig_macro.append(S_mac)
        if store:
            F_list.append(F)
            Sig_list.append(Sig)
        i, j = driving_component
        F_drv = F_mac[i, j]
        eng = F_drv - (1.0 if i == j else 0.0)
        if enable_console:
            print(f"step {s}/{n_steps}: F_{lbl}={F_drv:.5f}, eng_strain={eng:.5f}, Sig_{lbl}={S_mac[i, j] / 1e9:.4f} GPa")
        if log_f:
            log_f.write(f"{_dt.now().strftime('%Y-%m-%d %H:%M:%S'):<20} {_time.time() - t0:<12.3f} {s:<8} "
                        f"{F_drv:<14.6f} {eng:<20.6f} {S_mac[i, j] / 1e9:<18.6f}\n")
        if glog_f:
            glog_f.write(f"{s:<8} {F_mac[0, 0]:<12.6f} {F_mac[1, 1]:<12.6f} {F_mac[0, 1]:<12.6f} "
                         f"{F_mac[0, 0] - 1:<14.6f} {F_mac[1, 1] - 1:<14.6f} {P_mac[0, 0] / 1e9:<14.6f} "
                         f"{P_mac[1, 1] / 1e9:<14.6f} {P_mac[0, 1] / 1e9:<14.6f} {S_mac[0, 0] / 1e9:<16.6f} "
                         f"{S_mac[1, 1] / 1e9:<16.6f} {S_mac[0, 1] / 1e9:<16.6f}\n")
        if checkpoint_path is not None and (checkpoint_interval == "current" or (
                isinstance(checkpoint_interval, int) and s % checkpoint_interval == 0)):
            _checkpoint_2d(checkpoint_path if checkpoint_interval == "current" else f"{checkpoint_path}_{s:06d}", s,
                           E, nu, F, Sig, F_mac, S_mac, pixel)
        if vtk_path is not None:
            _vtk_step(vtk_interval, vtk_path, s, *_vtk_fields_2d(F, Sig), E, nu, pixel)
    if checkpoint_path is not None and (checkpoint_interval == "last" or (
            isinstance(checkpoint_interval, int) and n_steps % checkpoint_interval != 0)):
        _checkpoint_2d(f"{checkpoint_path}_final", n_steps, E, nu, F, Sig, F_macro[-1], Sig_macro[-1], pixel)
    if vtk_path is not None:
        _vtk_final(vtk_interval, vtk_path, n_steps, *_vtk_fields_2d(F, Sig), E, nu, pixel)
    if log_f:
        log_f.close()
    if glog_f:
        glog_f.close()
    return np.array(F_macro), np.array(Sig_macro), np.array(P_macro), F_list, Sig_list


def _vtk_fields_2d(F, Sig):
    """Green-Lagrange strain and Cauchy stress, spatial-first (:2797-2800)."""
    E_GL = 0.5 * (np.einsum("kixy,kjxy->ijxy", F, F) - np.eye(2)[:, :, None, None])
    return np.moveaxis(E_GL, (0, 1), (2, 3)), np.moveaxis(Sig, (0, 1), (2, 3))


def _checkpoint_2d(path, step, E, nu, F, Sig, F_mac, S_mac, pixel):
    """The reference's checkpoint of a 2D finite-strain step: Green-Lagrange
    strain and Cauchy stress, spatial-first (nx, ny, 2, 2)."""
    from . import checkpoint as C
    E_GL = 0.5 * (np.einsum("kixy,kjxy->ijxy", F, F) - np.eye(2)[:, :, None, None])
    C.save_checkpoint_2d(path, step, E, nu, np.moveaxis(E_GL, (0, 1), (2, 3)), np.moveaxis(Sig, (0, 1), (2, 3)),
                         F_mac, S_mac, pixel)
