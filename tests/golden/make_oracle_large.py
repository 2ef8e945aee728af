"""Oracle outputs at the finite-strain sizes the GPU kernels specialise for.

The warp-line finite-strain passes run for sides 64, 96 and 128; the numpy
oracle (oracle/fs.py, pinned to the reference by tests/golden/fs3d_*.npz)
needs minutes per load step there, so its results are computed once here and
committed as small fixtures: the fields F and P at 4096 seeded voxels, their
means and Frobenius norms over the whole grid, and the macro deformation.

    python tests/golden/make_oracle_large.py            # all
    python tests/golden/make_oracle_large.py fs3d_64     # one

Cases (Neo-Hookean with F_p on 2 % of voxels, the finite-strain workload's
material at that side):
  * fs3d_64  -- one mixed-BC load step: F_xx = 1.005 prescribed, lateral mean
    Cauchy stresses driven to zero (tol_macro 1e3 Pa), Newton 1e-10, CG 1e-11;
  * fs3d_96  -- one Newton solve at the prescribed F_bar = diag(1.005, 0.998,
    0.998) (no stress-controlled components), Newton 1e-10, CG 1e-11.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.abspath(os.path.join(HERE, "..", "..")))

from oracle import fs as OF  # noqa: E402
from mgkmc_b200 import workloads as W  # noqa: E402

N_SAMPLE = 4096


def sample_index(n, seed):
    return np.sort(np.random.default_rng(seed).choice(n ** 3, size=N_SAMPLE, replace=False))


def summarise(F, P, Sig, idx):
    """F, P, Sig spatial-first (n, n, n, 3, 3)."""
    Fs, Ps = F.reshape(-1, 9), P.reshape(-1, 9)
    return dict(idx=idx, F_s=Fs[idx], P_s=Ps[idx], F_mean=Fs.mean(axis=0), P_mean=Ps.mean(axis=0),
                Sig_mean=Sig.reshape(-1, 9).mean(axis=0), F_norm=np.linalg.norm(Fs - np.eye(3).ravel()),
                P_norm=np.linalg.norm(Ps), F_max=np.max(np.abs(Fs - np.eye(3).ravel())), P_max=np.max(np.abs(Ps)))


def fs3d_64():
    n = 64
    E, nu, Fp = W.fs3d_material(n, n, n, np.random.default_rng(64))
    F0 = np.broadcast_to(np.eye(3), (n, n, n, 3, 3)).copy()
    Fb, _, Pt, Pm = OF.build_bc_3d((0, 0), 0.005, {(1, 1): 0.0, (2, 2): 0.0})
    t = time.perf_counter()
    F, P, Sig, Fbo = OF.solver_step_3d(F0, Fb, E, nu, OF.to_spatial(Fp), (0, 0), Pt, Pm, tol_NW=1e-10,
                                       tol_CG=1e-11, max_NW=40, tol_macro=1e3, max_iter_macro=40,
                                       model="neo_hookean", krylov="cg")
    print(f"fs3d_64: {time.perf_counter() - t:.0f} s")
    np.savez_compressed(os.path.join(HERE, "fs3d_neohookean_64_oracle.npz"), F_bar_in=Fb, F_bar_out=Fbo, P_mask=Pm,
                        **summarise(F, P, Sig, sample_index(n, 640)))


def fs3d_96():
    n = 96
    E, nu, Fp = W.fs3d_material(n, n, n, np.random.default_rng(96))
    F0 = np.broadcast_to(np.eye(3), (n, n, n, 3, 3)).copy()
    Fb = np.diag([1.005, 0.998, 0.998])
    t = time.perf_counter()
    F, P, Sig, Fbo = OF.solver_step_3d(F0, Fb, E, nu, OF.to_spatial(Fp), (0, 0), None, None, tol_NW=1e-10,
                                       tol_CG=1e-11, max_NW=40, model="neo_hookean", krylov="cg")
    print(f"fs3d_96: {time.perf_counter() - t:.0f} s")
    np.savez_compressed(os.path.join(HERE, "fs3d_neohookean_96_oracle.npz"), F_bar_in=Fb, F_bar_out=Fbo,
                        **summarise(F, P, Sig, sample_index(n, 960)))


if __name__ == "__main__":
    for name in (sys.argv[1:] or ("fs3d_64", "fs3d_96")):
        globals()[name]()
