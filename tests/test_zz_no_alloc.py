"""The allocation-free 2D LS entry point (mgk_ls2d_solve_noalloc).

It serves callers that cannot allocate device memory -- a host application
whose caching allocator already owns the GPU's memory, a serving process with
a fixed memory budget, code that must not trigger cudaFree's device-wide
synchronisation.  Its scratch lives in one file-scope device array shared by
every call, so these tests check that two calls in a row (different problems,
sizes and start modes) each reproduce the plan-based entry point
(mgk_ls2d_create + mgk_ls2d_solve) within the LS tolerance, and that grids
above the array's maximum are refused with a clear error.  This file runs
last so that a failure here does not hide the other GPU tests; it also passes
alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from mgkmc_b200 import _lib as L
from mgkmc_b200 import workloads as W

pytestmark = pytest.mark.gpu
TOL = 1e-9


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _noalloc(E, nu, ep, eb, eps_init, max_iter, tol, plane_mode=0):
    import torch
    nx, ny = E.shape
    d = torch.device("cuda")
    tE, tnu = torch.from_numpy(E).to(d), torch.from_numpy(nu).to(d)
    tep = torch.from_numpy(ep).to(d) if ep is not None else None
    tin = torch.from_numpy(eps_init).to(d) if eps_init is not None else None
    eps = torch.empty((nx, ny, 2, 2), dtype=torch.float64, device=d)
    sig = torch.empty_like(eps)
    info = L.LsInfo()
    ebc = (ctypes.c_double * 4)(*np.asarray(eb, dtype=np.float64).ravel())
    rc = L.lib().mgk_ls2d_solve_noalloc(nx, ny, plane_mode, L.ptr(tE), L.ptr(tnu), L.ptr(tep), ebc, L.ptr(tin),
                                        L.ptr(eps), L.ptr(sig), max_iter, tol, ctypes.byref(info), L.stream_ptr())
    return rc, eps.cpu().numpy(), sig.cpu().numpy(), info


def _plan(E, nu, ep, eb, eps_init, max_iter, tol, plane_mode="plane_strain"):
    import torch
    from mgkmc_b200.linear_elastic_simulator import Ls2dSolver
    nx, ny = E.shape
    d = torch.device("cuda")
    s = Ls2dSolver(nx, ny, plane_mode)
    s.set_material(torch.from_numpy(E).to(d), torch.from_numpy(nu).to(d),
                   torch.from_numpy(ep).to(d) if ep is not None else None)
    eps = torch.empty((nx, ny, 2, 2), dtype=torch.float64, device=d)
    sig = torch.empty_like(eps)
    tin = torch.from_numpy(eps_init).to(d) if eps_init is not None else None
    info = s.solve(eb, eps, sig, eps_init=tin, max_iter=max_iter, tol=tol)
    return eps.cpu().numpy(), sig.cpu().numpy(), info.iterations


def test_noalloc_matches_plan_entry_point_on_consecutive_calls():
    # call 1: 256x256 cold start; call 2: 96x64 warm start, asymmetric eps_bar,
    # plane stress -- the second call must not see anything the first left behind
    E1, nu1, ep1, eb1 = W.ls2d_problem(256, 256, seed=21)
    rng = np.random.default_rng(22)
    E2, nu2 = W.ls2d_material(96, 64, rng)
    ep2 = W.pure_shear_eigenstrain_2d(96, 64, rng)
    eb2 = np.array([[0.004, 0.002], [-0.001, -0.003]])
    init2 = 1e-3 * rng.standard_normal((96, 64, 2, 2))
    rc1, e1, s1, i1 = _noalloc(E1, nu1, ep1, eb1, None, 300, 1e-10)
    rc2, e2, s2, i2 = _noalloc(E2, nu2, ep2, eb2, init2, 300, 1e-10, plane_mode=1)
    assert rc1 == L.OK and rc2 == L.OK, L.lib().mgk_last_error()
    pe1, ps1, it1 = _plan(E1, nu1, ep1, eb1, None, 300, 1e-10)
    pe2, ps2, it2 = _plan(E2, nu2, ep2, eb2, init2, 300, 1e-10, plane_mode="plane_stress")
    assert rel(e1, pe1) < TOL and rel(s1, ps1) < TOL
    assert rel(e2, pe2) < TOL and rel(s2, ps2) < TOL
    assert i1.iterations == it1 and i2.iterations == it2
    # a third call repeats the first problem: same answer again
    rc3, e3, s3, i3 = _noalloc(E1, nu1, ep1, eb1, None, 300, 1e-10)
    assert rc3 == L.OK and rel(e3, pe1) < TOL and rel(s3, ps1) < TOL


def test_noalloc_rejects_grids_above_its_maximum():
    lib = L.lib()
    info = L.LsInfo()
    eb = (ctypes.c_double * 4)(0.01, 0, 0, 0)
    rc = lib.mgk_ls2d_solve_noalloc(512, 512, 0, None, None, None, eb, None, None, None, 10, 1e-6,
                                    ctypes.byref(info), L.stream_ptr())
    assert rc == L.BAD_ARG
    assert b"exceeds the maximum" in lib.mgk_last_error()
