"""GPU parity of the 3D LS solver (mgk_ls3d_*) against the reference's golden
outputs and the oracle; tolerance 1e-9 relative (max-abs over the field)."""
import numpy as np
import pytest

from mgkmc_b200 import workloads as W
from oracle import ls as OL

pytestmark = pytest.mark.gpu
TOL = 1e-9


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("name", ["ls3d_8x8x8", "ls3d_12x8x6"])
def test_golden(golden, name):
    from mgkmc_b200.linear_elastic_simulator import spectral_solver_3d
    g = golden(name)
    eps, sig, _, _ = spectral_solver_3d(g["E"], g["nu"], g["eps_bar"], g["eps_plastic"], max_iter=2, tol=0.0)
    assert rel(eps, g["eps_it2"]) < TOL
    assert rel(sig, g["sig_it2"]) < TOL
    eps, sig, em, sm = spectral_solver_3d(g["E"], g["nu"], g["eps_bar"], g["eps_plastic"], max_iter=300, tol=1e-10)
    assert rel(eps, g["eps_conv"]) < TOL
    assert rel(sig, g["sig_conv"]) < TOL


@pytest.mark.parametrize("shape", [(32, 32, 32), (24, 16, 12), (64, 48, 32), (8, 6, 1), (6, 9, 3), (64, 64, 64),
                                   (96, 64, 128)])
def test_oracle_sizes(shape):
    from mgkmc_b200.linear_elastic_simulator import spectral_solver_3d
    rng = np.random.default_rng(sum(shape))
    E, nu = W.ls3d_material(*shape, rng)
    ep = W.pure_shear_eigenstrain_3d(*shape, rng)
    eb = np.zeros((3, 3)); eb[0, 0] = 0.01; eb[0, 1] = 0.003; eb[1, 0] = -0.001
    o = OL.spectral_solver(E, nu, eb, ep, max_iter=200, tol=1e-10, return_info=True)
    eps, sig, em, sm = spectral_solver_3d(E, nu, eb, ep, max_iter=200, tol=1e-10)
    assert rel(eps, o[0]) < TOL and rel(sig, o[1]) < TOL


def test_warm_start_and_batch():
    import torch
    from mgkmc_b200.linear_elastic_simulator import Ls3dBatch
    sizes = [(16, 16, 16), (24, 24, 12)]
    rng = np.random.default_rng(5)
    probs = []
    for s in sizes:
        E, nu = W.ls3d_material(*s, rng)
        probs.append((E, nu, W.pure_shear_eigenstrain_3d(*s, rng)))
    B = Ls3dBatch(sizes)
    outs, sigs = [], []
    for r, (E, nu, ep) in enumerate(probs):
        B.set_material(r, torch.from_numpy(E).cuda(), torch.from_numpy(nu).cuda(), torch.from_numpy(ep).cuda())
        outs.append(torch.empty(E.shape + (3, 3), dtype=torch.float64, device="cuda"))
        sigs.append(torch.empty_like(outs[-1]))
    eb = np.diag([0.01, -0.002, 0.0])
    B.solve([0, 1], [eb, eb], outs, sigs, max_iter=200, tol=1e-10)
    for r, (E, nu, ep) in enumerate(probs):
        o = OL.spectral_solver(E, nu, eb, ep, max_iter=200, tol=1e-10)
        assert rel(outs[r].cpu().numpy(), o[0]) < TOL
    init = [o.clone() for o in outs]
    eb2 = eb + np.array([[0, 1e-3, 0], [0, 0, 0], [0, 0, 1e-3]])
    B.solve([1], [eb2], [outs[1]], [sigs[1]], eps_init=[init[1]], max_iter=200, tol=1e-10)
    E, nu, ep = probs[1]
    o = OL.spectral_solver(E, nu, eb2, ep, max_iter=200, tol=1e-10, eps_init=init[1].cpu().numpy())
    assert rel(outs[1].cpu().numpy(), o[0]) < TOL


def test_barrier_physics_homogeneous_units():
    # the reference's tests/test_barrier_physics.py:49-98 case: 16x16x1,
    # homogeneous E = 70 GPa, nu = 0.3, eps_xx = 1 %: sigma_xx = (lam + 2 mu) eps
    from mgkmc_b200.linear_elastic_simulator import spectral_solver_3d
    E = np.full((16, 16, 1), 70e9); nu = np.full((16, 16, 1), 0.3)
    eb = np.zeros((3, 3)); eb[0, 0] = 0.01
    eps, sig, em, sm = spectral_solver_3d(E, nu, eb, max_iter=50, tol=1e-6)
    lam = 70e9 * 0.3 / ((1 + 0.3) * (1 - 0.6)); mu = 70e9 / 2.6
    assert abs(sm[0, 0] - (lam + 2 * mu) * 0.01) < 1e-6 * (lam + 2 * mu) * 0.01


def test_warp_line_batch_matches_single_plans():
    # a batch of warp-line replicas (sides 64/96/128) against one-replica plans
    import torch
    from mgkmc_b200.linear_elastic_simulator import Ls3dBatch
    sizes = [(64, 64, 64), (96, 64, 128), (64, 128, 96)]
    rng = np.random.default_rng(9)
    probs = []
    for sh in sizes:
        E, nu = W.ls3d_material(*sh, rng)
        probs.append((E, nu, W.pure_shear_eigenstrain_3d(*sh, rng)))
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    eb = np.zeros((3, 3)); eb[0, 0] = 0.01
    B = Ls3dBatch(sizes)
    outs = []
    for r, (E, nu, ep) in enumerate(probs):
        B.set_material(r, t(E), t(nu), t(ep))
        outs.append(torch.empty(E.shape + (3, 3), dtype=torch.float64, device="cuda"))
    sigs = [torch.empty_like(o) for o in outs]
    B.solve(list(range(3)), [eb] * 3, outs, sigs, max_iter=200, tol=1e-10)
    for r, (E, nu, ep) in enumerate(probs):
        S = Ls3dBatch([sizes[r]])
        S.set_material(0, t(E), t(nu), t(ep))
        o1 = torch.empty_like(outs[r]); s1 = torch.empty_like(outs[r])
        S.solve([0], [eb], [o1], [s1], max_iter=200, tol=1e-10)
        assert rel(outs[r].cpu().numpy(), o1.cpu().numpy()) < 1e-12


@pytest.mark.parametrize("sizes", [[(64, 64, 64)], [(64, 96, 128), (64, 64, 64)]])
def test_mixed_precision_matches_fp64(sizes):
    # FP32 phase then FP64 to the same tolerance: converged fields agree with
    # the FP64 solve within the mixed form's bound (1e-6; ~1e-8 in practice)
    import torch
    from mgkmc_b200.linear_elastic_simulator import Ls3dBatch
    rng = np.random.default_rng(21)
    probs = []
    for sh in sizes:
        E, nu = W.ls3d_material(*sh, rng)
        probs.append((E, nu, W.pure_shear_eigenstrain_3d(*sh, rng)))
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    eb = np.zeros((3, 3)); eb[0, 0] = 0.01; eb[1, 2] = 0.002
    res = {}
    for prec in ("fp64", "mixed"):
        B = Ls3dBatch(sizes, precision=prec)
        outs = []
        for r, (E, nu, ep) in enumerate(probs):
            B.set_material(r, t(E), t(nu), t(ep))
            outs.append(torch.empty(E.shape + (3, 3), dtype=torch.float64, device="cuda"))
        sigs = [torch.empty_like(o) for o in outs]
        infos = B.solve(list(range(len(sizes))), [eb] * len(sizes), outs, sigs, max_iter=300, tol=1e-8)
        assert all(i.status == 0 for i in infos)
        res[prec] = [(o.cpu().numpy(), g.cpu().numpy()) for o, g in zip(outs, sigs)]
    for (e64, s64), (e32, s32) in zip(res["fp64"], res["mixed"]):
        assert rel(e32, e64) < 1e-6 and rel(s32, s64) < 1e-6


@pytest.mark.parametrize("tag", ["a", "b", "warm"])
def test_golden_secant(golden, tag):
    # 3D secant-degradation law (CTA-wide passes at 12 x 8 x 6) against the reference
    from mgkmc_b200.linear_elastic_simulator import spectral_solver_secant_3d
    g = golden("ls3d_secant_12x8x6")
    if tag == "warm":
        eps, sig, _, sm = spectral_solver_secant_3d(g["lam"], g["mu"], 0.3, 50.0, g["eps_bar"] * 1.1,
                                                    g["eps_plastic"], max_iter=500, tol=1e-12,
                                                    eps_init=g["eps_init"])
    else:
        eps, sig, _, sm = spectral_solver_secant_3d(g["lam"], g["mu"], float(g[f"d_{tag}"]), float(g[f"k_{tag}"]),
                                                    g["eps_bar"], g["eps_plastic"], max_iter=500, tol=1e-12)
    assert rel(eps, g[f"eps_{tag}"]) < TOL
    assert rel(sig, g[f"sig_{tag}"]) < TOL
    assert np.allclose(sm, g[f"sig_{tag}"].mean(axis=(0, 1, 2)), rtol=1e-9, atol=1e-3)


@pytest.mark.parametrize("shape,d,k", [((64, 64, 64), 0.5, 100.0), ((32, 24, 16), 0.8, 200.0),
                                       ((32, 24, 16), 0.0, 10.0)])
def test_secant_against_oracle(shape, d, k):
    # warp-line FP64 kernels (64^3) and the CTA-wide passes with the secant law,
    # against the oracle; d = 0 is Hooke's law with the (mean lam, mean mu) medium
    from mgkmc_b200.linear_elastic_simulator import spectral_solver_secant_3d
    rng = np.random.default_rng(sum(shape) + int(k))
    E, nu = W.ls3d_material(*shape, rng)
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    ep = W.pure_shear_eigenstrain_3d(*shape, rng, frac=0.1)
    eb = np.zeros((3, 3)); eb[0, 0] = 0.02; eb[1, 1] = -0.005; eb[0, 1] = 0.004; eb[1, 0] = 0.001
    o = OL.spectral_solver_secant_3d(lam, mu, d, k, eb, ep, max_iter=500, tol=1e-10)
    eps, sig, _, _ = spectral_solver_secant_3d(lam, mu, d, k, eb, ep, max_iter=500, tol=1e-10)
    assert rel(eps, o[0]) < TOL and rel(sig, o[1]) < TOL


def test_secant_refused_on_mixed_plans():
    from mgkmc_b200 import _lib as L
    from mgkmc_b200.linear_elastic_simulator import Ls3dBatch
    b = Ls3dBatch([(64, 64, 64)], precision="mixed")
    with pytest.raises(L.MgkError):
        b.set_secant(0.5, 100.0)
