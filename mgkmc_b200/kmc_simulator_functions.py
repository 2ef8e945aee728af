"""Drop-in per-voxel STZ/KMC kernels backed by the CUDA library.

Same names, arguments and in-place semantics as
mgkmc/kmc_simulator_functions.py (numpy arrays in and out).  Each call
stages its arrays on the current CUDA device, runs the ``mgk_kmc*`` kernels
and writes the results back into the caller's numpy arrays.  ``KmcDevice2D``
is the device-resident form (torch CUDA tensors, no host round trips) used by
the GPU KMC driver.

Selection draws: the reference's numba ``select_event_2d`` draws from numba's
private generator (kmc_simulator_functions.py:62), which ``np.random.seed``
does not seed.  This drop-in draws ``u`` from numpy's global generator,
exactly like the reference's pure-Python body ``select_event_2d.py_func``,
and ``select_event_2d_u`` takes the draw explicitly.
"""
import ctypes

import numpy as np

from . import _lib as L


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("mgkmc_b200 needs a CUDA device (no CPU fallback)")
    return torch


def _dev(a, torch, dtype=None):
    a = np.ascontiguousarray(a, dtype=dtype or np.float64)
    return torch.from_numpy(a).cuda()


def compute_barrier_2d(Q_field, Q0_field, sigma_field, catalog, volume, soft_prop, last_event_time, current_time,
                       prev_strain_dir, softening_cap, softening_scheme_idx=0, tau=np.inf):
    """In-place barrier update (kmc_simulator_functions.py:100-160)."""
    torch = _torch()
    nx, ny, M = Q_field.shape
    tQ = torch.empty((nx, ny, M), dtype=torch.float64, device="cuda")
    tQ0, ts, tc = _dev(Q0_field, torch), _dev(sigma_field, torch), _dev(catalog, torch)
    tsp, tl = _dev(soft_prop, torch), _dev(last_event_time, torch)
    tp = _dev(prev_strain_dir, torch) if int(softening_scheme_idx) == 1 else None
    L.check(L.lib().mgk_kmc2d_barrier(nx, ny, M, L.ptr(tQ), L.ptr(tQ0), L.ptr(ts), L.ptr(tc), float(volume),
                                      L.ptr(tsp), L.ptr(tl), float(current_time), L.ptr(tp), float(softening_cap),
                                      int(softening_scheme_idx), float(tau), L.stream_ptr()), "mgk_kmc2d_barrier")
    Q_field[...] = tQ.cpu().numpy()


def compute_rates_2d(Q_field, volume, temperature, nu0=1e13, cascade_mode=True):
    """(rates, indices, total_rate) (kmc_simulator_functions.py:5-56)."""
    torch = _torch()
    nx, ny, M = Q_field.shape
    n = nx * ny * M
    tQ = _dev(Q_field, torch)
    if isinstance(temperature, (int, float, np.number)):
        tT, Ts = None, float(temperature)
    else:
        tT, Ts = _dev(np.broadcast_to(np.asarray(temperature, dtype=np.float64), (nx, ny)), torch), 0.0
    rates = torch.empty(n, dtype=torch.float64, device="cuda")
    idx = torch.empty(n, dtype=torch.int64, device="cuda")
    prefix = torch.empty(n, dtype=torch.float64, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    tot = torch.zeros(1, dtype=torch.float64, device="cuda")
    work = torch.empty(int(L.lib().mgk_kmc_rates_work_bytes(n)), dtype=torch.uint8, device="cuda")
    L.check(L.lib().mgk_kmc2d_rates(nx, ny, M, L.ptr(tQ), float(volume), L.ptr(tT), Ts, float(nu0),
                                    1 if cascade_mode else 0, L.ptr(rates), L.ptr(idx), L.ptr(prefix), L.ptr(cnt),
                                    L.ptr(tot), L.ptr(work), L.stream_ptr()), "mgk_kmc2d_rates")
    c = int(cnt.item())
    return rates[:c].cpu().numpy(), idx[:c].cpu().numpy(), float(tot.item())


def select_event_2d_u(rates, total_rate, u):
    """First i with the sequential running sum >= u * total_rate
    (kmc_simulator_functions.py:58-67) for an explicit draw u in [0, 1)."""
    torch = _torch()
    rates = np.ascontiguousarray(rates, dtype=np.float64)
    n = rates.size
    tr = _dev(rates, torch) if n else torch.zeros(1, dtype=torch.float64, device="cuda")
    prefix = torch.empty(max(n, 1), dtype=torch.float64, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    tot = torch.zeros(1, dtype=torch.float64, device="cuda")
    L.check(L.lib().mgk_kmc_prefix(L.ptr(tr), n, L.ptr(prefix), L.ptr(cnt), L.ptr(tot), L.stream_ptr()),
            "mgk_kmc_prefix")
    tot.fill_(float(total_rate))  # the caller's total decides r, as in the reference
    out = torch.empty(1, dtype=torch.int64, device="cuda")
    L.check(L.lib().mgk_kmc_select(L.ptr(prefix), L.ptr(cnt), L.ptr(tot), float(u), L.ptr(out), L.stream_ptr()),
            "mgk_kmc_select")
    return int(out.item())


def select_event_2d(rates, total_rate):
    if total_rate <= 0:
        return -1
    return select_event_2d_u(rates, total_rate, np.random.random_sample())


def decode_index_2d(flat_idx, ny, M):
    """(x, y, m) of a flat mode index (kmc_simulator_functions.py:69-76)."""
    m = flat_idx % M
    t = flat_idx // M
    return t // ny, t % ny, m


def apply_flip_soa_2d(eps_plastic_field, soft_prop_field, last_event_time_field, catalog, x, y, m, current_time,
                      jp, jt, g_max, jn_frac):
    """In-place flip bookkeeping (kmc_simulator_functions.py:183-218)."""
    torch = _torch()
    nx, ny = eps_plastic_field.shape[:2]
    M = catalog.shape[2]
    te, ts, tl, tc = (_dev(eps_plastic_field, torch), _dev(soft_prop_field, torch), _dev(last_event_time_field, torch),
                      _dev(catalog, torch))
    L.check(L.lib().mgk_kmc2d_flip(nx, ny, M, L.ptr(te), L.ptr(ts), L.ptr(tl), L.ptr(tc), int(x), int(y), int(m),
                                   float(current_time), float(jp), float(jt), float(g_max), float(jn_frac),
                                   L.stream_ptr()), "mgk_kmc2d_flip")
    eps_plastic_field[...] = te.cpu().numpy()
    soft_prop_field[...] = ts.cpu().numpy()
    last_event_time_field[...] = tl.cpu().numpy()
