"""Drop-in 3D STZ/KMC kernels backed by the CUDA library.

Same names, arguments and in-place semantics as mgkmc/stz/barriers.py
(``compute_barrier``), mgkmc/stz/kmc.py (``compute_rates``,
``select_event``, ``decode_index``) and mgkmc/stz/cascade.py
(``apply_flip_soa``).  Selection draws come from numpy's global generator
(the reference's numba generator is not seedable from numpy), and
``select_event_u`` takes the draw explicitly.
"""
import numpy as np

from . import _lib as L
from .kmc_simulator_functions import _dev, _torch, select_event_2d_u


def compute_barrier(Q_field, Q0_field, sigma_field, catalog, volume, soft_prop, last_event_time, current_time,
                    prev_strain_dir, softening_cap, softening_scheme_idx=0, tau=np.inf):
    """In-place barrier update (mgkmc/stz/barriers.py:4-100)."""
    torch = _torch()
    nx, ny, nz, M = Q_field.shape
    tQ = torch.empty((nx, ny, nz, M), dtype=torch.float64, device="cuda")
    tQ0, ts, tc = _dev(Q0_field, torch), _dev(sigma_field, torch), _dev(catalog, torch)
    tsp, tl = _dev(soft_prop, torch), _dev(last_event_time, torch)
    tp = _dev(prev_strain_dir, torch) if int(softening_scheme_idx) == 1 else None
    L.check(L.lib().mgk_kmc3d_barrier(nx, ny, nz, M, L.ptr(tQ), L.ptr(tQ0), L.ptr(ts), L.ptr(tc), float(volume),
                                      L.ptr(tsp), L.ptr(tl), float(current_time), L.ptr(tp), float(softening_cap),
                                      int(softening_scheme_idx), float(tau), L.stream_ptr()), "mgk_kmc3d_barrier")
    Q_field[...] = tQ.cpu().numpy()


def compute_rates(Q_field, volume, temperature, nu0=1e13, cascade_mode=True):
    """(rates, indices, total_rate) (mgkmc/stz/kmc.py:4-74)."""
    torch = _torch()
    nx, ny, nz, M = Q_field.shape
    n = nx * ny * nz * M
    tQ = _dev(Q_field, torch)
    if isinstance(temperature, (int, float, np.number)):
        tT, Ts = None, float(temperature)
    else:
        tT, Ts = _dev(np.broadcast_to(np.asarray(temperature, dtype=np.float64), (nx, ny, nz)), torch), 0.0
    rates = torch.empty(n, dtype=torch.float64, device="cuda")
    idx = torch.empty(n, dtype=torch.int64, device="cuda")
    prefix = torch.empty(n, dtype=torch.float64, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    tot = torch.zeros(1, dtype=torch.float64, device="cuda")
    work = torch.empty(int(L.lib().mgk_kmc_rates_work_bytes(n)), dtype=torch.uint8, device="cuda")
    L.check(L.lib().mgk_kmc3d_rates(nx, ny, nz, M, L.ptr(tQ), float(volume), L.ptr(tT), Ts, float(nu0),
                                    1 if cascade_mode else 0, L.ptr(rates), L.ptr(idx), L.ptr(prefix), L.ptr(cnt),
                                    L.ptr(tot), L.ptr(work), L.stream_ptr()), "mgk_kmc3d_rates")
    c = int(cnt.item())
    return rates[:c].cpu().numpy(), idx[:c].cpu().numpy(), float(tot.item())


def select_event_u(rates, total_rate, u):
    """mgkmc/stz/kmc.py:76-92 with an explicit draw."""
    return select_event_2d_u(rates, total_rate, u)


def select_event(rates, total_rate):
    if total_rate <= 0:
        return -1
    return select_event_u(rates, total_rate, np.random.random_sample())


def decode_index(flat_idx, ny, nz, M):
    """(x, y, z, m) of a flat mode index (mgkmc/stz/kmc.py:94-103)."""
    m = flat_idx % M
    t = flat_idx // M
    z = t % nz
    t = t // nz
    return t // ny, t % ny, z, m


def apply_flip_soa(eps_plastic_field, key_field, soft_prop_field, last_event_time_field, catalog, x, y, z, m,
                   current_time, jp, jt, g_max, jn_frac):
    """In-place flip bookkeeping (mgkmc/stz/cascade.py:43-111; key_field unused, as there)."""
    torch = _torch()
    nx, ny, nz = eps_plastic_field.shape[:3]
    M = catalog.shape[3]
    te, ts, tl, tc = (_dev(eps_plastic_field, torch), _dev(soft_prop_field, torch), _dev(last_event_time_field, torch),
                      _dev(catalog, torch))
    L.check(L.lib().mgk_kmc3d_flip(nx, ny, nz, M, L.ptr(te), L.ptr(ts), L.ptr(tl), L.ptr(tc), int(x), int(y), int(z),
                                   int(m), float(current_time), float(jp), float(jt), float(g_max), float(jn_frac),
                                   L.stream_ptr()), "mgk_kmc3d_flip")
    eps_plastic_field[...] = te.cpu().numpy()
    soft_prop_field[...] = ts.cpu().numpy()
    last_event_time_field[...] = tl.cpu().numpy()
