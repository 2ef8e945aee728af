"""numpy restatement of the per-voxel STZ / KMC kernels (oracle).

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).

Follows mgkmc/kmc_simulator_functions.py (2D) and mgkmc/stz/{barriers,kmc,
cascade}.py (3D).  The restatement keeps the reference's floating-point
operation order where it matters for bit-exactness:
  * contractions are left-to-right sums starting from 0.0 over (i, j) in C
    order (kmc_simulator_functions.py:136-157);
  * the total rate is the sequential left-to-right FP64 sum in (x, y[, z], m)
    order (:36-55), i.e. ``np.add.accumulate`` whose last element is the total;
  * selection returns the first i with S_i >= u * total (:58-67), where
    ``u * total`` is exactly numpy's ``uniform(0, total)`` for the draw u.
"""
import numpy as np

KB = 8.617e-5             # eV/K (kmc_simulator_functions.py:23)
GPA_NM3_TO_EV = 6.241509  # (:108)


def _seq_contract(a, b, d):
    """sum_ij a[..., i, j] * b[..., i, j] accumulated left to right from 0.0."""
    acc = np.zeros(np.broadcast_shapes(a.shape[:-2], b.shape[:-2]))
    for i in range(d):
        for j in range(d):
            acc = acc + a[..., i, j] * b[..., i, j]
    return acc


def _softening_base(soft_prop, last_event_time, current_time, cap, tau):
    # kmc_simulator_functions.py:114-128 ; stz/barriers.py:33-53
    g_t = soft_prop[..., 1]
    t_last = last_event_time
    g_t_curr = np.zeros_like(g_t)
    pos = g_t > 0
    if tau == np.inf:
        g_t_curr = np.where(pos, g_t, 0.0)
    else:
        dt = np.maximum(current_time - t_last, 0.0)
        with np.errstate(invalid="ignore", over="ignore"):
            decayed = g_t * np.exp(-dt / tau)
        g_t_curr = np.where(pos & (t_last != -np.inf), decayed, 0.0)
    g_base = soft_prop[..., 0] + g_t_curr
    if cap > 0:
        g_base = np.where(g_base > cap, cap, g_base)
    return g_base


def compute_barrier(Q, Q0, sig, catalog, volume, soft_prop, last_event_time, current_time,
                    prev_dir, cap, scheme=0, tau=np.inf):
    """In-place barrier update, 2D or 3D (d from sig's last axis).

    2D: kmc_simulator_functions.py:100-160.  3D: stz/barriers.py:4-100.
    """
    d = sig.shape[-1]
    g_base = _softening_base(soft_prop, last_event_time, current_time, cap, tau)[..., None]
    if scheme == 1:
        dot = _seq_contract(catalog, prev_dir[..., None, :, :], d)
        nm = _seq_contract(catalog, catalog, d)
        npv = _seq_contract(prev_dir, prev_dir, d)[..., None]
        norm_m = np.sqrt(nm)
        norm_p = np.sqrt(npv)
        small = (norm_p < 1e-12) | (norm_m < 1e-12)
        with np.errstate(invalid="ignore", divide="ignore"):
            c = dot / (norm_m * norm_p)
        mod = np.where(small, 1.0, (1.0 + c) * (1.0 + c) / 4.0)
    else:
        mod = 1.0
    g_eff = mod * g_base
    w_sum = _seq_contract(sig[..., None, :, :], catalog, d)
    w_val = 0.5 * volume * (w_sum / 1e9) * GPA_NM3_TO_EV
    Q[...] = Q0 * np.exp(-g_eff) - w_val
    return Q


def compute_rates(Q, volume, temperature, nu0=1e13, cascade_mode=True):
    """(rates, indices, total) -- kmc_simulator_functions.py:5-56 ; stz/kmc.py:4-74."""
    M = Q.shape[-1]
    T = np.broadcast_to(np.asarray(temperature, dtype=np.float64), Q.shape[:-1])
    with np.errstate(divide="ignore"):
        beta = np.where(T > 0.0, 1.0 / (KB * np.where(T > 0.0, T, 1.0)), np.inf)
    q = Q.reshape(-1)
    b = np.repeat(beta.reshape(-1), M)
    with np.errstate(invalid="ignore", over="ignore"):
        r = np.where(q <= 0, volume * nu0, volume * nu0 * np.exp(-q * b))
    idx = np.arange(q.size, dtype=np.int64)
    if cascade_mode:
        keep = q > 0
        r, idx = r[keep], idx[keep]
    total = float(np.add.accumulate(r)[-1]) if r.size else 0.0
    return r, idx, total


def select_event(rates, total_rate, u):
    """First i with S_i >= u*total (S sequential); -1 if total <= 0 (:58-67)."""
    if total_rate <= 0:
        return -1
    r = 0.0 + (total_rate - 0.0) * u
    S = np.add.accumulate(rates)
    i = int(np.searchsorted(S, r, side="left"))
    return i if i < len(rates) else len(rates) - 1


def select_event_loop(rates, total_rate, u):
    """Literal sequential restatement (small inputs only)."""
    if total_rate <= 0:
        return -1
    r = 0.0 + (total_rate - 0.0) * u
    s = 0.0
    for i in range(len(rates)):
        s += rates[i]
        if s >= r:
            return i
    return len(rates) - 1


def decode_index_2d(flat, ny, M):
    # kmc_simulator_functions.py:69-76
    m = flat % M
    t = flat // M
    return t // ny, t % ny, m


def decode_index_3d(flat, ny, nz, M):
    # stz/kmc.py:94-103
    m = flat % M
    t = flat // M
    z = t % nz
    t = t // nz
    return t // ny, t % ny, z, m


def apply_flip_2d(eps_p, soft, t_last, catalog, x, y, m, t, jp, jt, gmax, jn):
    """kmc_simulator_functions.py:183-218 (in place)."""
    nx, ny = eps_p.shape[:2]
    eps_p[x, y] += catalog[x, y, m]
    e11, e22, e12 = catalog[x, y, m, 0, 0], catalog[x, y, m, 1, 1], catalog[x, y, m, 0, 1]
    s = e12 ** 2 + (e22 ** 2 + e11 ** 2 + (e11 - e22) ** 2) / 6.0
    gp = soft[x, y, 0] + jp * s
    if gmax > 0 and gp > gmax:
        gp = gmax
    soft[x, y, 0] = gp
    soft[x, y, 1] = jt * s
    t_last[x, y] = t
    if jn > 0.0:
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                if dx == 0 and dy == 0:
                    continue
                a, b = (x + dx + nx) % nx, (y + dy + ny) % ny
                g = soft[a, b, 0] + jn * jp * s
                if gmax > 0 and g > gmax:
                    g = gmax
                soft[a, b, 0] = g
                soft[a, b, 1] += jn * jt * s


def apply_flip_3d(eps_p, soft, t_last, catalog, x, y, z, m, t, jp, jt, gmax, jn):
    """stz/cascade.py:43-111 (in place)."""
    nx, ny, nz = eps_p.shape[:3]
    eps_p[x, y, z] += catalog[x, y, z, m]
    c = catalog[x, y, z, m]
    e11, e22, e33, e12, e13, e23 = c[0, 0], c[1, 1], c[2, 2], c[0, 1], c[0, 2], c[1, 2]
    s = (e12 ** 2 + e23 ** 2 + e13 ** 2) + ((e22 - e33) ** 2 + (e33 - e11) ** 2 + (e11 - e22) ** 2) / 6.0
    gp = soft[x, y, z, 0] + jp * s
    if gmax > 0 and gp > gmax:
        gp = gmax
    soft[x, y, z, 0] = gp
    soft[x, y, z, 1] = jt * s
    t_last[x, y, z] = t
    if jn > 0.0:
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    if dx == 0 and dy == 0 and dz == 0:
                        continue
                    a, b, cc = (x + dx + nx) % nx, (y + dy + ny) % ny, (z + dz + nz) % nz
                    g = soft[a, b, cc, 0] + jn * jp * s
                    if gmax > 0 and g > gmax:
                        g = gmax
                    soft[a, b, cc, 0] = g
                    soft[a, b, cc, 1] = soft[a, b, cc, 1] + jn * jt * s


def find_unstable_2d(Q, threshold=0.0):
    """(x, y, m) rows of the modes with Q < threshold, in (x, y, m) order
    (mgkmc/kmc_simulator_functions.py:162-181)."""
    nx, ny, M = Q.shape
    flat = np.flatnonzero(Q.reshape(-1) < threshold)
    return np.stack([flat // (ny * M), (flat // M) % ny, flat % M], axis=1).astype(np.int64)
