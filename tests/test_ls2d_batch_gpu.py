"""Batched (ragged, one launch per stage) and mixed-precision 2D LS solves.

* a ragged batch reproduces each replica's single-plan solve (same kernels,
  same per-replica reductions: equal to 1e-12);
* replicas converge independently (different iteration counts in one batch);
* subsets of slots can be solved while the other slots keep their state;
* the mixed form (FP32 bulk, FP64 finish) reaches the requested update norm
  and stays within 1e-6 relative field error of the FP64 oracle.
"""
import numpy as np
import pytest

from mgkmc_b200 import workloads as W
from oracle import ls as OL

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _t(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


SIZES = [(256, 256), (128, 128), (192, 192), (96, 64), (64, 64), (384, 128)]


def _problems(sizes, seed0=100):
    return [W.ls2d_problem(nx, ny, seed=seed0 + i) for i, (nx, ny) in enumerate(sizes)]


@pytest.mark.parametrize("sizes", [SIZES, [(768, 64), (64, 64), (256, 128), (1024, 96)]])
def test_ragged_batch_matches_single_plans(sizes):
    # the second set runs every replica through the two-warp-line kernel
    # variant (a side above 512 in the plan); single plans of the small ones
    # use the one-warp variant: same arithmetic, same bits
    import torch
    from mgkmc_b200.linear_elastic_simulator import Ls2dBatch, Ls2dSolver
    SIZES = sizes
    probs = _problems(SIZES)
    B = Ls2dBatch(SIZES)
    outs, sigs = [], []
    for r, (E, nu, ep, eb) in enumerate(probs):
        B.set_material(r, _t(E), _t(nu), _t(ep))
        outs.append(torch.empty(E.shape + (2, 2), dtype=torch.float64, device="cuda"))
        sigs.append(torch.empty_like(outs[-1]))
    infos = B.solve(list(range(len(SIZES))), [p[3] for p in probs], outs, sigs, max_iter=300, tol=1e-10)
    iters = [i.iterations for i in infos]
    for r, (E, nu, ep, eb) in enumerate(probs):
        s = Ls2dSolver(*SIZES[r])
        s.set_material(_t(E), _t(nu), _t(ep))
        e1 = torch.empty_like(outs[r]); s1 = torch.empty_like(outs[r])
        info = s.solve(eb, e1, s1, max_iter=300, tol=1e-10)
        assert info.iterations == iters[r]
        assert rel(outs[r].cpu().numpy(), e1.cpu().numpy()) < 1e-12
        assert rel(sigs[r].cpu().numpy(), s1.cpu().numpy()) < 1e-12
    # the largest replica against the oracle
    E, nu, ep, eb = probs[0]
    o = OL.spectral_solver(E, nu, eb, ep, max_iter=300, tol=1e-10)
    assert rel(outs[0].cpu().numpy(), o[0]) < 1e-9


def test_subset_selection_and_warm_start():
    import torch
    from mgkmc_b200.linear_elastic_simulator import Ls2dBatch
    sizes = [(64, 64), (128, 96), (64, 64)]
    probs = _problems(sizes, seed0=7)
    B = Ls2dBatch(sizes)
    outs = []
    for r, (E, nu, ep, eb) in enumerate(probs):
        B.set_material(r, _t(E), _t(nu), _t(ep))
        outs.append(torch.empty(E.shape + (2, 2), dtype=torch.float64, device="cuda"))
    sig = [torch.empty_like(o) for o in outs]
    B.solve([2, 0], [probs[2][3], probs[0][3]], [outs[2], outs[0]], [sig[2], sig[0]], max_iter=300, tol=1e-10)
    B.solve([1], [probs[1][3]], [outs[1]], [sig[1]], max_iter=300, tol=1e-10)
    for r, (E, nu, ep, eb) in enumerate(probs):
        o = OL.spectral_solver(E, nu, eb, ep, max_iter=300, tol=1e-10)
        assert rel(outs[r].cpu().numpy(), o[0]) < 1e-9, r
    # warm start replica 1 from its own solution at a new macro strain
    eb2 = np.array([[0.012, 0.001], [0.001, -0.002]])
    E, nu, ep, _ = probs[1]
    init = outs[1].clone()
    B.solve([1], [eb2], [outs[1]], [sig[1]], eps_init=[init], max_iter=300, tol=1e-10)
    o = OL.spectral_solver(E, nu, eb2, ep, max_iter=300, tol=1e-10, eps_init=init.cpu().numpy())
    assert rel(outs[1].cpu().numpy(), o[0]) < 1e-9


@pytest.mark.parametrize("nx,ny", [(256, 256), (192, 192), (128, 64)])
def test_mixed_precision_accuracy(nx, ny):
    import torch
    from mgkmc_b200.linear_elastic_simulator import Ls2dBatch, Ls2dSolver
    E, nu, ep, eb = W.ls2d_problem(nx, ny, seed=42)
    o = OL.spectral_solver(E, nu, eb, ep, max_iter=500, tol=1e-13)
    M = Ls2dBatch([(nx, ny)], precision="mixed")
    M.set_material(0, _t(E), _t(nu), _t(ep))
    eps = torch.empty((nx, ny, 2, 2), dtype=torch.float64, device="cuda")
    sig = torch.empty_like(eps)
    info = M.solve([0], [eb], [eps], [sig], max_iter=300, tol=1e-8)[0]
    assert info.status == 0 and info.final_diff < 1e-8
    assert rel(eps.cpu().numpy(), o[0]) < 1e-6
    assert rel(sig.cpu().numpy(), o[1]) < 1e-6
    # equilibrium residual of the mixed result: one FP64 iteration from it
    S = Ls2dSolver(nx, ny)
    S.set_material(_t(E), _t(nu), _t(ep))
    chk = S.solve(eb, torch.empty_like(eps), torch.empty_like(eps), eps_init=eps, max_iter=1, tol=0.0)
    assert chk.final_diff < 1e-8


def test_mixed_batch_many_replicas():
    import torch
    from mgkmc_b200.linear_elastic_simulator import Ls2dBatch
    sizes = [(128, 128)] * 12 + [(192, 192)] * 4
    probs = _problems(sizes, seed0=300)
    M = Ls2dBatch(sizes, precision="mixed")
    outs = []
    for r, (E, nu, ep, eb) in enumerate(probs):
        M.set_material(r, _t(E), _t(nu), _t(ep))
        outs.append(torch.empty(E.shape + (2, 2), dtype=torch.float64, device="cuda"))
    infos = M.solve(list(range(len(sizes))), [p[3] for p in probs], outs, [None] * len(sizes), max_iter=300,
                    tol=1e-8)
    for r in (0, 7, 13, 15):
        E, nu, ep, eb = probs[r]
        o = OL.spectral_solver(E, nu, eb, ep, max_iter=500, tol=1e-13)
        assert infos[r].status == 0
        assert rel(outs[r].cpu().numpy(), o[0]) < 1e-6


def test_autotune_and_every_family_agree():
    # the autotuner picks among the kernel families that can serve the plan;
    # every family computes the same solves (same radix schedules, different
    # work decomposition; the compiler may contract FP32 operations
    # differently per kernel, so agreement is to 1e-10, far inside tol)
    import torch
    from mgkmc_b200.linear_elastic_simulator import Ls2dBatch
    sizes = [(128, 128), (96, 64), (128, 96)]
    probs = _problems(sizes, seed0=300)
    ref = None
    for family in (None, 256, 512, 1024, 0):
        B = Ls2dBatch(sizes, precision="mixed")
        for r, (E, nu, ep, eb) in enumerate(probs):
            B.set_material(r, _t(E), _t(nu), _t(ep))
        if family is None:
            fam, ms = B.autotune([0, 1, 2], [p[3] for p in probs], n=3)
            assert fam in (0, 256, 512, 1024) and ms > 0
            for r, (E, nu, ep, eb) in enumerate(probs):  # iterates were used for timing
                B.set_material(r, _t(E), _t(nu), _t(ep))
        else:
            B.set_family(family)
        outs = [torch.empty(p[0].shape + (2, 2), dtype=torch.float64, device="cuda") for p in probs]
        sigs = [torch.empty_like(o) for o in outs]
        infos = B.solve([0, 1, 2], [p[3] for p in probs], outs, sigs, max_iter=300, tol=1e-10)
        got = [o.cpu().numpy() for o in outs]
        if ref is None:
            ref = got
        for a, b in zip(got, ref):
            assert rel(a, b) < 1e-10
