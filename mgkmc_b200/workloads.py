"""Seeded synthetic inputs for the mechanical-equilibrium workloads.

The reference publishes no benchmark dataset; these generators restate the
material, eigenstrain and barrier models of the five benchmark workloads:

* ``ls2d_material``    -- 2D heterogeneous isotropic medium: per-voxel shear
  modulus mu = mu0 (1 + 0.1 N(0,1)) clipped to [0.7, 1.3] mu0 (mu0 = 33.3 GPa),
  bulk modulus K = 100 GPa, converted to the (E, nu) pair the reference API
  takes (E = 9 K mu / (3K + mu), nu = (3K - 2 mu) / (2 (3K + mu))).
* ``pure_shear_eigenstrain_2d`` -- pure-shear STZ eigenstrains of magnitude
  gamma0 on a fraction of voxels chosen uniformly, orientation theta ~ U[0, pi):
  eps_p = (gamma0/2) [[cos 2t, sin 2t], [sin 2t, -cos 2t]] (the gamma0/2 tensor
  amplitude of mgkmc/kmc_simulator_functions.py:85-90).
* ``kmc2d_state``      -- per-voxel STZ catalog of M pure-shear modes and
  Gaussian barriers Q0 ~ N(1.0, 0.15) eV clipped below at 0.3 eV (the
  reference clips, mgkmc/kmc_simulator_functions.py:226-227).
* ``fs3d_material``    -- 3D log-normal shear modulus (mean 33.3 GPa, CV 0.1),
  K = 100 GPa, and plastic eigen-deformations F_p = I + 0.05 S on 2 % of voxels
  (S traceless symmetric with unit Frobenius norm).

All arrays are float64 numpy arrays in the reference layouts: (nx, ny) moduli,
(nx, ny, 2, 2) strain/stress (AoS, C order), tensor-first (3, 3, nx, ny, nz)
for finite strain.
"""
import numpy as np

MU0 = 33.3e9
K_BULK = 100e9


def e_nu_from_k_mu(K, mu):
    E = 9.0 * K * mu / (3.0 * K + mu)
    nu = (3.0 * K - 2.0 * mu) / (2.0 * (3.0 * K + mu))
    return E, nu


def ls2d_material(nx, ny, rng, mu0=MU0, K=K_BULK, cv=0.1):
    mu = mu0 * (1.0 + cv * rng.standard_normal((nx, ny)))
    mu = np.clip(mu, 0.7 * mu0, 1.3 * mu0)
    Kf = np.full((nx, ny), float(K))
    return e_nu_from_k_mu(Kf, mu)


def pure_shear_eigenstrain_2d(nx, ny, rng, frac=0.05, gamma0=0.1):
    N = nx * ny
    nsel = int(round(frac * N))
    sel = rng.choice(N, size=nsel, replace=False)
    theta = rng.uniform(0.0, np.pi, size=nsel)
    c, s = np.cos(2 * theta), np.sin(2 * theta)
    ep = np.zeros((N, 2, 2))
    ep[sel, 0, 0] = 0.5 * gamma0 * c
    ep[sel, 1, 1] = -0.5 * gamma0 * c
    ep[sel, 0, 1] = 0.5 * gamma0 * s
    ep[sel, 1, 0] = 0.5 * gamma0 * s
    return ep.reshape(nx, ny, 2, 2)


def ls2d_problem(nx, ny, seed, frac=0.05, gamma0=0.1, eps_xx=0.01):
    """One heterogeneous 2D LS problem: (E, nu, eps_plastic, eps_bar)."""
    rng = np.random.default_rng(seed)
    E, nu = ls2d_material(nx, ny, rng)
    ep = pure_shear_eigenstrain_2d(nx, ny, rng, frac, gamma0)
    eps_bar = np.zeros((2, 2))
    eps_bar[0, 0] = eps_xx
    return E, nu, ep, eps_bar


def kmc2d_state(nx, ny, M, rng, gamma0=0.1, q_mean=1.0, q_std=0.15, q_min=0.3):
    """STZ catalog (nx, ny, M, 2, 2) and barriers Q0 (nx, ny, M)."""
    theta = rng.uniform(0.0, np.pi, size=(nx, ny, M))
    c, s = np.cos(2 * theta), np.sin(2 * theta)
    cat = np.empty((nx, ny, M, 2, 2))
    cat[..., 0, 0] = 0.5 * gamma0 * c
    cat[..., 1, 1] = -0.5 * gamma0 * c
    cat[..., 0, 1] = 0.5 * gamma0 * s
    cat[..., 1, 0] = 0.5 * gamma0 * s
    Q0 = np.clip(rng.normal(q_mean, q_std, size=(nx, ny, M)), q_min, None)
    return cat, Q0


def ls3d_material(nx, ny, nz, rng, mu0=MU0, K=K_BULK, cv=0.1):
    mu = mu0 * (1.0 + cv * rng.standard_normal((nx, ny, nz)))
    mu = np.clip(mu, 0.7 * mu0, 1.3 * mu0)
    return e_nu_from_k_mu(np.full((nx, ny, nz), float(K)), mu)


def pure_shear_eigenstrain_3d(nx, ny, nz, rng, frac=0.05, gamma0=0.1):
    """In-plane pure-shear eigenstrains (the glass catalog of mgkmc/stz/catalog.py:8-29)."""
    N = nx * ny * nz
    nsel = int(round(frac * N))
    sel = rng.choice(N, size=nsel, replace=False)
    theta = rng.uniform(0.0, np.pi, size=nsel)
    c, s = np.cos(2 * theta), np.sin(2 * theta)
    ep = np.zeros((N, 3, 3))
    ep[sel, 0, 0] = 0.5 * gamma0 * c
    ep[sel, 1, 1] = -0.5 * gamma0 * c
    ep[sel, 0, 1] = 0.5 * gamma0 * s
    ep[sel, 1, 0] = 0.5 * gamma0 * s
    return ep.reshape(nx, ny, nz, 3, 3)


def fs3d_material(nx, ny, nz, rng, mu_mean=MU0, cv=0.1, K=K_BULK, fp_frac=0.02, fp_amp=0.05):
    """3D finite-strain material: (E, nu) fields and tensor-first F_p (3,3,nx,ny,nz)."""
    s2 = np.log(1.0 + cv * cv)
    m = np.log(mu_mean) - 0.5 * s2
    mu = np.exp(m + np.sqrt(s2) * rng.standard_normal((nx, ny, nz)))
    E, nu = e_nu_from_k_mu(np.full((nx, ny, nz), float(K)), mu)
    N = nx * ny * nz
    Fp = np.zeros((N, 3, 3))
    Fp[:, 0, 0] = Fp[:, 1, 1] = Fp[:, 2, 2] = 1.0
    nsel = int(round(fp_frac * N))
    sel = rng.choice(N, size=nsel, replace=False)
    G = rng.standard_normal((nsel, 3, 3))
    S = 0.5 * (G + G.transpose(0, 2, 1))
    tr = np.trace(S, axis1=1, axis2=2)
    S -= tr[:, None, None] / 3.0 * np.eye(3)[None]
    S /= np.sqrt(np.sum(S * S, axis=(1, 2)))[:, None, None]
    Fp[sel] += fp_amp * S
    Fp = Fp.reshape(nx, ny, nz, 3, 3)
    return E, nu, np.ascontiguousarray(np.moveaxis(Fp, (3, 4), (0, 1)))


# ------------------------------------------------ device-side generators ---
# The serving layer builds each request's inputs on the GPU from the
# request's seed (torch's CUDA generator): same distributions as the numpy
# generators above, different draws.  Host generation of a 1024^2 catalog
# would take longer than its solves.

def _gen(seed, device):
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    return g


def ls2d_problem_dev(nx, ny, seed, device, frac=0.05, gamma0=0.1, eps_xx=0.01, mu0=MU0, K=K_BULK, cv=0.1):
    """(E, nu, eps_plastic, eps_bar) with E, nu (nx, ny) and eps_plastic
    (nx, ny, 2, 2) float64 tensors on ``device``."""
    import torch
    g = _gen(seed, device)
    f64 = torch.float64
    mu = mu0 * (1.0 + cv * torch.randn((nx, ny), generator=g, device=device, dtype=f64))
    mu = mu.clamp(0.7 * mu0, 1.3 * mu0)
    E = 9.0 * K * mu / (3.0 * K + mu)
    nu = (3.0 * K - 2.0 * mu) / (2.0 * (3.0 * K + mu))
    N = nx * ny
    nsel = int(round(frac * N))
    sel = torch.randperm(N, generator=g, device=device)[:nsel]
    theta = torch.rand(nsel, generator=g, device=device, dtype=f64) * np.pi
    c, s = torch.cos(2 * theta), torch.sin(2 * theta)
    ep = torch.zeros((N, 2, 2), dtype=f64, device=device)
    ep[sel, 0, 0] = 0.5 * gamma0 * c
    ep[sel, 1, 1] = -0.5 * gamma0 * c
    ep[sel, 0, 1] = 0.5 * gamma0 * s
    ep[sel, 1, 0] = 0.5 * gamma0 * s
    eps_bar = np.zeros((2, 2))
    eps_bar[0, 0] = eps_xx
    return E, nu, ep.reshape(nx, ny, 2, 2), eps_bar


def kmc2d_state_dev(nx, ny, M, seed, device, gamma0=0.1, q_mean=1.0, q_std=0.15, q_min=0.3):
    """STZ catalog (nx, ny, M, 2, 2) and barriers Q0 (nx, ny, M) on ``device``."""
    import torch
    g = _gen(seed + 7919, device)
    f64 = torch.float64
    theta = torch.rand((nx, ny, M), generator=g, device=device, dtype=f64) * np.pi
    c, s = torch.cos(2 * theta), torch.sin(2 * theta)
    cat = torch.empty((nx, ny, M, 2, 2), dtype=f64, device=device)
    cat[..., 0, 0] = 0.5 * gamma0 * c
    cat[..., 1, 1] = -0.5 * gamma0 * c
    cat[..., 0, 1] = 0.5 * gamma0 * s
    cat[..., 1, 0] = 0.5 * gamma0 * s
    Q0 = (q_mean + q_std * torch.randn((nx, ny, M), generator=g, device=device, dtype=f64)).clamp_min(q_min)
    return cat, Q0


def fs3d_material_dev(nx, ny, nz, seed, device, mu_mean=MU0, cv=0.1, K=K_BULK, fp_frac=0.02, fp_amp=0.05):
    """(lam, mu) (nx, ny, nz) and tensor-first F_p (3, 3, nx, ny, nz) on ``device``."""
    import torch
    g = _gen(seed, device)
    f64 = torch.float64
    s2 = np.log(1.0 + cv * cv)
    m = np.log(mu_mean) - 0.5 * s2
    mu = torch.exp(m + np.sqrt(s2) * torch.randn((nx, ny, nz), generator=g, device=device, dtype=f64))
    E = 9.0 * K * mu / (3.0 * K + mu)
    nu = (3.0 * K - 2.0 * mu) / (2.0 * (3.0 * K + mu))
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu2 = E / (2 * (1 + nu))
    N = nx * ny * nz
    Fp = torch.zeros((N, 3, 3), dtype=f64, device=device)
    Fp[:, 0, 0] = 1.0
    Fp[:, 1, 1] = 1.0
    Fp[:, 2, 2] = 1.0
    nsel = int(round(fp_frac * N))
    sel = torch.randperm(N, generator=g, device=device)[:nsel]
    G = torch.randn((nsel, 3, 3), generator=g, device=device, dtype=f64)
    S = 0.5 * (G + G.transpose(1, 2))
    tr = S.diagonal(dim1=1, dim2=2).sum(-1)
    S = S - tr[:, None, None] / 3.0 * torch.eye(3, dtype=f64, device=device)[None]
    S = S / torch.sqrt((S * S).sum(dim=(1, 2)))[:, None, None]
    Fp[sel] += fp_amp * S
    Fp = Fp.reshape(nx, ny, nz, 3, 3).permute(3, 4, 0, 1, 2).contiguous()
    return lam.contiguous(), mu2.contiguous(), Fp


def ls3d_material_dev(nx, ny, nz, seed, device, mu0=MU0, K=K_BULK, cv=0.1):
    """3D (E, nu) (nx, ny, nz) on ``device``: the 2D workloads' medium in 3D."""
    import torch
    g = _gen(seed, device)
    f64 = torch.float64
    mu = mu0 * (1.0 + cv * torch.randn((nx, ny, nz), generator=g, device=device, dtype=f64))
    mu = mu.clamp(0.7 * mu0, 1.3 * mu0)
    E = 9.0 * K * mu / (3.0 * K + mu)
    nu = (3.0 * K - 2.0 * mu) / (2.0 * (3.0 * K + mu))
    return E.contiguous(), nu.contiguous()


def kmc3d_state_dev(nx, ny, nz, M, seed, device, gamma0=0.1, q_mean=1.0, q_std=0.15, q_min=0.3):
    """In-plane pure-shear STZ catalog (nx, ny, nz, M, 3, 3) and barriers Q0
    (nx, ny, nz, M) on ``device`` (the 2D catalog's distribution, glass modes
    of mgkmc/stz/catalog.py:7-29 with fixed amplitude gamma0/2)."""
    import torch
    g = _gen(seed + 7919, device)
    f64 = torch.float64
    theta = torch.rand((nx, ny, nz, M), generator=g, device=device, dtype=f64) * np.pi
    c, s = torch.cos(2 * theta), torch.sin(2 * theta)
    cat = torch.zeros((nx, ny, nz, M, 3, 3), dtype=f64, device=device)
    cat[..., 0, 0] = 0.5 * gamma0 * c
    cat[..., 1, 1] = -0.5 * gamma0 * c
    cat[..., 0, 1] = 0.5 * gamma0 * s
    cat[..., 1, 0] = 0.5 * gamma0 * s
    Q0 = (q_mean + q_std * torch.randn((nx, ny, nz, M), generator=g, device=device, dtype=f64)).clamp_min(q_min)
    return cat, Q0
