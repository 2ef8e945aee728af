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

Host traffic per call:
  * ``apply_flip_soa_2d`` is O(1) work and moves O(1) bytes: the flipped
    voxel's 3 x 3 periodic neighbourhood (its voxel alone when the neighbour
    fraction is zero) is gathered, updated on the device and scattered back;
  * ``compute_rates_2d`` returns the rates as a read-only array that keeps the
    device running sums of that call, so ``select_event_2d`` on it uploads
    nothing and only searches on the device (a writable or foreign rates
    array is uploaded and summed, as before);
  * ``compute_barrier_2d`` uploads its inputs each call unless device mirrors
    are enabled (``use_device_mirrors(True)``): then catalog, Q0,
    prev_strain_dir, soft_prop and last_event_time stay on the device, keyed
    on the numpy buffers, and only the voxels flipped through
    ``apply_flip_soa_2d`` since the previous call are re-read from the host.
    That is exact when the caller changes these arrays only at flipped
    voxels, as the reference's drivers do (flip bookkeeping, then the redraw
    of the flipped voxel's catalog and barriers, kmc_simulator.py:1025-1042);
    ``clear_device_mirrors()`` drops them after any other change.
"""
import ctypes
import weakref

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


# ------------------------------------------------------------ mirrors ---
_MIRRORS = {}        # key of a numpy buffer -> (weak reference to the array, device tensor)
_DIRTY = {}          # key of a mirrored buffer -> voxels (x, y) to re-read
_USE_MIRRORS = [False]


def use_device_mirrors(on=True):
    """Keep compute_barrier_2d's large inputs on the device between calls
    (exact when the caller changes them only at voxels flipped through
    apply_flip_soa_2d, as the reference's drivers do)."""
    _USE_MIRRORS[0] = bool(on)
    if not on:
        clear_device_mirrors()


def clear_device_mirrors():
    _MIRRORS.clear()
    _DIRTY.clear()


def _key(a):
    return (a.__array_interface__["data"][0], a.shape, a.dtype.str, a.strides)


def _mirror(a, torch):
    """Device copy of numpy array ``a``: uploaded on first use, then refreshed
    at the voxels (leading two indices) marked dirty since the last use."""
    k = _key(a)
    ent = _MIRRORS.get(k)
    if ent is None or ent[0]() is not a:
        # first use, or a different array now at the same address
        t = _dev(a, torch)
        _MIRRORS[k] = (weakref.ref(a), t)
        _DIRTY[k] = set()
        return t
    t = ent[1]
    dirty = _DIRTY.get(k)
    if dirty:
        xs = np.fromiter((v[0] for v in dirty), dtype=np.int64)
        ys = np.fromiter((v[1] for v in dirty), dtype=np.int64)
        vals = torch.from_numpy(np.ascontiguousarray(a[xs, ys], dtype=np.float64)).cuda()
        t[torch.from_numpy(xs).cuda(), torch.from_numpy(ys).cuda()] = vals
        dirty.clear()
    return t


def _mark_dirty(arrays, voxels):
    for a in arrays:
        k = _key(a)
        if k in _DIRTY:
            _DIRTY[k].update(voxels)


def compute_barrier_2d(Q_field, Q0_field, sigma_field, catalog, volume, soft_prop, last_event_time, current_time,
                       prev_strain_dir, softening_cap, softening_scheme_idx=0, tau=np.inf):
    """In-place barrier update (kmc_simulator_functions.py:100-160)."""
    torch = _torch()
    nx, ny, M = Q_field.shape
    tQ = torch.empty((nx, ny, M), dtype=torch.float64, device="cuda")
    up = _mirror if _USE_MIRRORS[0] else _dev
    tQ0, ts, tc = up(Q0_field, torch), _dev(sigma_field, torch), up(catalog, torch)
    tsp, tl = up(soft_prop, torch), up(last_event_time, torch)
    tp = up(prev_strain_dir, torch) if int(softening_scheme_idx) == 1 else None
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
    out = rates[:c].cpu().numpy().view(_Rates)
    out._mgk = (prefix, cnt, tot)  # the device running sums of this call
    out.flags.writeable = False
    idx_h = np.arange(c, dtype=np.int64) if not cascade_mode else idx[:c].cpu().numpy()
    return out, idx_h, float(tot.item())


class _Rates(np.ndarray):
    """Read-only rates that keep the device running sums they were built with."""

    def __array_finalize__(self, obj):
        self._mgk = None


def select_event_2d_u(rates, total_rate, u):
    """First i with the sequential running sum >= u * total_rate
    (kmc_simulator_functions.py:58-67) for an explicit draw u in [0, 1)."""
    torch = _torch()
    dev = getattr(rates, "_mgk", None)
    if isinstance(rates, _Rates) and dev is not None and not rates.flags.writeable:
        prefix, cnt, _ = dev  # running sums of the compute_rates_2d call that made these rates
        tot = torch.full((1,), float(total_rate), dtype=torch.float64, device="cuda")
    else:
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
    """In-place flip bookkeeping (kmc_simulator_functions.py:183-218).  Only
    the voxels the flip can touch cross PCIe: the flipped voxel, or its 3 x 3
    periodic neighbourhood when jn_frac > 0 (the whole fields on grids
    narrower than 3, where the neighbourhood wraps onto itself)."""
    torch = _torch()
    nx, ny = eps_plastic_field.shape[:2]
    M = catalog.shape[2]
    x, y, m = int(x), int(y), int(m)
    if jn_frac > 0.0 and (nx < 3 or ny < 3):
        xs, ys, w, cx, cy = np.arange(nx), np.arange(ny), (nx, ny), x, y
    elif jn_frac > 0.0:
        xs, ys, w, cx, cy = (x + np.arange(-1, 2)) % nx, (y + np.arange(-1, 2)) % ny, (3, 3), 1, 1
    else:
        xs, ys, w, cx, cy = np.array([x]), np.array([y]), (1, 1), 0, 0
    ix = np.ix_(xs, ys)
    te, ts, tl = (_dev(eps_plastic_field[ix], torch), _dev(soft_prop_field[ix], torch),
                  _dev(last_event_time_field[ix], torch))
    cat = np.zeros((w[0], w[1], M, 2, 2))
    cat[cx, cy] = catalog[x, y]
    tc = _dev(cat, torch)
    L.check(L.lib().mgk_kmc2d_flip(w[0], w[1], M, L.ptr(te), L.ptr(ts), L.ptr(tl), L.ptr(tc), cx, cy, m,
                                   float(current_time), float(jp), float(jt), float(g_max), float(jn_frac),
                                   L.stream_ptr()), "mgk_kmc2d_flip")
    eps_plastic_field[ix] = te.cpu().numpy()
    soft_prop_field[ix] = ts.cpu().numpy()
    last_event_time_field[ix] = tl.cpu().numpy()
    if _USE_MIRRORS[0]:
        # the flipped voxel's catalog, barriers and previous direction are
        # redrawn by the caller next; the neighbourhood's softening changed here
        vox = {(int(a), int(b)) for a in xs for b in ys}
        _mark_dirty((soft_prop_field, last_event_time_field), vox)
        _mark_dirty_catalog((x, y))


def _mark_dirty_catalog(voxel):
    """Marks the flipped voxel in every mirrored buffer whose leading axes are
    a grid: the caller's redraws of catalog, Q0 and prev_strain_dir land there
    (kmc_simulator.py:1030-1042) before the next barrier update."""
    for k, d in _DIRTY.items():
        d.add(voxel)
