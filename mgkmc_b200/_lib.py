"""ctypes binding of libmgkmc_cuda.so (the C-ABI declared in include/mgkmc.h).

The library is the only compute path: there is no CPU fallback.  Loading
fails loudly when the shared object is missing or when no CUDA device is
present at call time.
"""
import ctypes
import os
import re
from ctypes import POINTER, Structure, c_char_p, c_double, c_int, c_int64, c_void_p

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmgkmc_cuda.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "mgkmc.h")

OK, NOT_CONVERGED, NONFINITE, BAD_ARG, OOM, TIMEOUT, CUDA_ERROR = range(7)
PLANE_STRAIN, PLANE_STRESS = 0, 1
FP64, MIXED = 0, 1


class MgkError(RuntimeError):
    def __init__(self, status, where, msg):
        self.status = status
        super().__init__(f"{where}: status {status} ({_STATUS.get(status, '?')}): {msg}")


_STATUS = {0: "ok", 1: "not converged", 2: "non-finite", 3: "bad argument", 4: "out of memory",
           5: "timeout", 6: "CUDA error"}


class LsInfo(Structure):
    _fields_ = [("iterations", c_int), ("status", c_int), ("final_diff", c_double),
                ("eps_mean", c_double * 4), ("sig_mean", c_double * 4)]


class LsInfo3(Structure):
    _fields_ = [("iterations", c_int), ("status", c_int), ("final_diff", c_double),
                ("eps_mean", c_double * 9), ("sig_mean", c_double * 9)]


class FsInfo(Structure):
    _fields_ = [("newton_iterations", c_int), ("krylov_iterations", c_int), ("macro_iterations", c_int),
                ("status", c_int), ("max_stress_error", c_double), ("sig_mean", c_double * 9)]


_P = c_void_p
_SIGS = {
    "mgk_version": (c_int, []),
    "mgk_status_string": (c_char_p, [c_int]),
    "mgk_last_error": (c_char_p, []),
    "mgk_fft_supported": (c_int, [c_int]),
    "mgk_ls2d_create": (c_int, [c_int, c_int, c_int, c_int, POINTER(c_void_p)]),
    "mgk_ls2d_destroy": (c_int, [_P]),
    "mgk_ls2d_set_material": (c_int, [_P, _P, _P, _P, _P]),
    "mgk_ls2d_set_eigenstrain": (c_int, [_P, _P, _P]),
    "mgk_ls2d_create_batch": (c_int, [c_int, POINTER(c_int), POINTER(c_int), c_int, c_int, POINTER(c_void_p)]),
    "mgk_ls2d_set_material_rep": (c_int, [_P, c_int, _P, _P, _P, _P]),
    "mgk_ls2d_set_lame_rep": (c_int, [_P, c_int, _P, _P, _P, _P]),
    "mgk_ls2d_set_secant": (c_int, [_P, c_double, c_double]),
    "mgk_ls2d_set_rose": (c_int, [_P, c_double, c_double, c_int]),
    "mgk_ls2d_set_landau": (c_int, [_P, _P, c_int, c_double, c_double, c_double, c_int]),
    "mgk_ls2d_set_e33_out": (c_int, [_P, c_int, _P]),
    "mgk_ls2d_set_anderson": (c_int, [_P, c_int]),
    "mgk_aa_work_bytes": (c_int64, [c_int64]),
    "mgk_aa_update": (c_int, [c_int64, _P, _P, _P, c_int, c_int, c_int, c_int, _P, _P, _P]),
    "mgk_aa_mix": (c_int, [c_int64, _P, _P, c_int, c_int, _P, _P, _P]),
    "mgk_ls2d_set_eigenstrain_rep": (c_int, [_P, c_int, _P, _P]),
    "mgk_ls2d_autotune": (c_int, [_P, c_int, POINTER(c_int), POINTER(c_double), c_int, POINTER(c_int),
                                  POINTER(ctypes.c_float), _P]),
    "mgk_ls2d_set_family": (c_int, [_P, c_int]),
    "mgk_ls2d_collect": (c_int, [_P, c_int, POINTER(c_int), POINTER(LsInfo), _P]),
    "mgk_ls2d_solve_batch": (c_int, [_P, c_int, POINTER(c_int), POINTER(c_double), POINTER(c_void_p),
                                     POINTER(c_void_p), POINTER(c_void_p), c_int, c_double, POINTER(LsInfo), _P]),
    "mgk_ls2d_profile_batch": (c_int, [_P, c_int, POINTER(c_int), POINTER(c_double), c_int, c_int,
                                       POINTER(ctypes.c_float), POINTER(ctypes.c_float), _P]),
    "mgk_ls2d_solve": (c_int, [_P, POINTER(c_double), _P, _P, _P, c_int, c_double, POINTER(LsInfo), _P]),
    "mgk_ls2d_profile": (c_int, [_P, POINTER(c_double), c_int, POINTER(ctypes.c_float), POINTER(ctypes.c_float), _P]),
    "mgk_ls2d_solve_noalloc": (c_int, [c_int, c_int, c_int, _P, _P, _P, POINTER(c_double), _P, _P, _P, c_int,
                                       c_double, POINTER(LsInfo), _P]),
    "mgk_ls3d_create": (c_int, [c_int, c_int, c_int, POINTER(c_void_p)]),
    "mgk_ls3d_create_batch": (c_int, [c_int, POINTER(c_int), POINTER(c_int), POINTER(c_int), POINTER(c_void_p)]),
    "mgk_ls3d_set_precision": (c_int, [_P, c_int]),
    "mgk_ls3d_destroy": (c_int, [_P]),
    "mgk_ls3d_set_material_rep": (c_int, [_P, c_int, _P, _P, _P, _P]),
    "mgk_ls3d_set_eigenstrain_rep": (c_int, [_P, c_int, _P, _P]),
    "mgk_ls3d_set_lame_rep": (c_int, [_P, c_int, _P, _P, _P, _P]),
    "mgk_ls3d_set_landau": (c_int, [_P, _P, c_int, c_double, c_double, c_double]),
    "mgk_ls3d_set_secant": (c_int, [_P, c_double, c_double]),
    "mgk_ls3d_solve_batch": (c_int, [_P, c_int, POINTER(c_int), POINTER(c_double), POINTER(c_void_p),
                                     POINTER(c_void_p), POINTER(c_void_p), c_int, c_double, POINTER(LsInfo3), _P]),
    "mgk_fs3d_create": (c_int, [c_int, c_int, c_int, c_int, POINTER(c_void_p)]),
    "mgk_fs3d_destroy": (c_int, [_P]),
    "mgk_fs3d_set_precision": (c_int, [_P, c_int]),
    "mgk_fs3d_autotune": (c_int, [_P, c_int, POINTER(c_int), POINTER(ctypes.c_float), _P]),
    "mgk_fs3d_profile": (c_int, [_P, c_int, c_int, POINTER(ctypes.c_float), _P]),
    "mgk_fs3d_set_material": (c_int, [_P, _P, _P, _P, _P]),
    "mgk_fs3d_set_F": (c_int, [_P, _P, _P]),
    "mgk_fs3d_set_plane_strain": (c_int, [_P, c_int]),
    "mgk_fs3d_set_plane_stress": (c_int, [_P, c_int]),
    "mgk_fs3d_step": (c_int, [_P, POINTER(c_double), c_int, c_int, POINTER(c_double), POINTER(c_int), c_double,
                              c_double, c_double, c_double, c_int, c_double, c_int, POINTER(c_double),
                              POINTER(FsInfo), _P]),
    "mgk_fs3d_get": (c_int, [_P, _P, _P, _P, _P]),
    "mgk_kmc2d_barrier": (c_int, [c_int, c_int, c_int, _P, _P, _P, _P, c_double, _P, _P, c_double, _P,
                                  c_double, c_int, c_double, _P]),
    "mgk_kmc2d_barrier_total": (c_int, [c_int, c_int, c_int, _P, _P, _P, _P, c_double, _P, _P, c_double, _P,
                                        c_double, c_int, c_double, c_double, _P, c_double, c_double, _P, _P, _P]),
    "mgk_kmc_rates_work_bytes": (c_int64, [c_int64]),
    "mgk_kmc2d_rates": (c_int, [c_int, c_int, c_int, _P, c_double, _P, c_double, c_double, c_int, _P, _P, _P,
                                _P, _P, _P, _P]),
    "mgk_kmc_prefix": (c_int, [_P, c_int64, _P, _P, _P, _P]),
    "mgk_kmc_select": (c_int, [_P, _P, _P, c_double, _P, _P]),
    "mgk_kmc2d_flip": (c_int, [c_int, c_int, c_int, _P, _P, _P, _P, c_int, c_int, c_int, c_double, c_double,
                               c_double, c_double, c_double, _P]),
    "mgk_ls2d_sync_voxel": (c_int, [_P, c_int, _P, _P, _P]),
    "mgk_kmc_scan_work_bytes": (c_int64, [c_int64]),
    "mgk_kmc2d_rates_only": (c_int, [c_int, c_int, c_int, _P, c_double, _P, c_double, c_double, _P, _P]),
    "mgk_kmc_prefix_fast": (c_int, [_P, c_int64, _P, _P, _P, _P, _P]),
    "mgk_kmc2d_event": (c_int, [c_int, c_int, c_int, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, c_double, c_double,
                                c_double, c_double, c_double, _P, _P]),
    "mgk_kmc2d_patch_setup": (c_int, [c_int, c_int, c_int, _P, _P, _P, _P, _P]),
    "mgk_kmc2d_patch": (c_int, [c_int, c_int, c_int, _P, _P, c_double, _P, _P, c_int, _P, _P, _P, _P]),
    "mgk_kmc3d_barrier": (c_int, [c_int, c_int, c_int, c_int, _P, _P, _P, _P, c_double, _P, _P, c_double, _P,
                                  c_double, c_int, c_double, _P]),
    "mgk_kmc3d_rates": (c_int, [c_int, c_int, c_int, c_int, _P, c_double, _P, c_double, c_double, c_int, _P, _P,
                                _P, _P, _P, _P, _P]),
    "mgk_kmc3d_flip": (c_int, [c_int, c_int, c_int, c_int, _P, _P, _P, _P, c_int, c_int, c_int, c_int, c_double,
                               c_double, c_double, c_double, c_double, _P]),
    "mgk_kmc3d_event": (c_int, [c_int, c_int, c_int, c_int, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, c_double,
                                c_double, c_double, c_double, c_double, _P, _P]),
}

_lib = None


def declared_symbols(header=HEADER):
    """Names of every function declared in the public header."""
    text = open(header).read()
    return sorted(set(re.findall(r"MGK_API\s+[\w\s\*]+?\b(mgk_\w+)\s*\(", text)))


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m mgkmc_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in _SIGS.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def check(status, where, allow=(OK,)):
    if status in allow:
        return status
    msg = lib().mgk_last_error().decode(errors="replace")
    raise MgkError(status, where, msg)


def ptr(t):
    """Device address of a torch tensor (or None -> NULL)."""
    return None if t is None else c_void_p(t.data_ptr())


def stream_ptr(stream=None):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return c_void_p(s.cuda_stream)
