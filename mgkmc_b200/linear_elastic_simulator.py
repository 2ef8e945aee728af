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

import numpy as np

from . import _lib as L

_PLANE = {"plane_strain": L.PLANE_STRAIN, "plane_stress": L.PLANE_STRESS}


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("mgkmc_b200 needs a CUDA device (no CPU fallback)")
    return torch


class Ls2dSolver:
    """Plan-owning 2D LS solver on one device.

    Fields are torch float64 CUDA tensors in the reference layouts:
    E, nu (nx, ny); eps_plastic, eps, sig (nx, ny, 2, 2)."""

    def __init__(self, nx, ny, plane_mode="plane_strain", precision="fp64", device=None):
        torch = _torch()
        self.nx, self.ny = int(nx), int(ny)
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.plane_mode = plane_mode
        self.precision = precision
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            L.check(L.lib().mgk_ls2d_create(self.nx, self.ny, _PLANE[plane_mode],
                                            L.FP64 if precision == "fp64" else L.FP32, ctypes.byref(h)),
                    "mgk_ls2d_create")
        self._h = h
        self.info = L.LsInfo()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                L.lib().mgk_ls2d_destroy(h)
            except Exception:
                pass
            self._h = None

    def set_material(self, E, nu, eps_plastic=None, stream=None):
        self._E, self._nu, self._ep = E, nu, eps_plastic  # keep alive until the stream consumes them
        L.check(L.lib().mgk_ls2d_set_material(self._h, L.ptr(E), L.ptr(nu), L.ptr(eps_plastic),
                                              L.stream_ptr(stream)), "mgk_ls2d_set_material")

    def set_eigenstrain(self, eps_plastic, stream=None):
        self._ep = eps_plastic
        L.check(L.lib().mgk_ls2d_set_eigenstrain(self._h, L.ptr(eps_plastic), L.stream_ptr(stream)),
                "mgk_ls2d_set_eigenstrain")

    def solve(self, eps_bar, eps_out, sig_out, eps_init=None, max_iter=200, tol=1e-6, sync=True, stream=None):
        eb = (ctypes.c_double * 4)(*[float(v) for v in np.asarray(eps_bar, dtype=np.float64).reshape(4)])
        info = self.info if sync else None
        st = L.lib().mgk_ls2d_solve(self._h, eb, L.ptr(eps_init), L.ptr(eps_out), L.ptr(sig_out), int(max_iter),
                                    float(tol), ctypes.byref(info) if info is not None else None,
                                    L.stream_ptr(stream))
        L.check(st, "mgk_ls2d_solve", allow=(L.OK, L.NONFINITE))
        return info


    def profile_kernels(self, eps_bar, reps=50, stream=None):
        """Mean (row_ms, col_ms) of the two iteration kernels (CUDA events)."""
        eb = (ctypes.c_double * 4)(*[float(v) for v in np.asarray(eps_bar, dtype=np.float64).reshape(4)])
        r, c = ctypes.c_float(), ctypes.c_float()
        L.check(L.lib().mgk_ls2d_profile(self._h, eb, int(reps), ctypes.byref(r), ctypes.byref(c),
                                         L.stream_ptr(stream)), "mgk_ls2d_profile")
        return r.value, c.value


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
