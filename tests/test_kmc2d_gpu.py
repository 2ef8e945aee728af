"""GPU parity of the STZ/KMC kernels (mgk_kmc*) against the reference's golden
outputs and the oracle.  Selection index and flip bookkeeping are compared
bit for bit; barriers and rates to a few ulps (exp() differs by <= 1 ulp
between CUDA and the host libm)."""
import numpy as np
import pytest

from mgkmc_b200 import workloads as W
from oracle import kmc as OK

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def K():
    from mgkmc_b200 import kmc_simulator_functions as K
    return K


def test_barrier_golden(K, golden):
    g = golden("kmc2d_16x12")
    for c, (t, cap, scheme, tau, vol) in enumerate(g["cases"]):
        Q = np.zeros_like(g["Q0"])
        K.compute_barrier_2d(Q, g["Q0"], g["sig"], g["catalog"], vol, g["soft_prop"], g["last_event_time"], t,
                             g["prev_dir"], cap, int(scheme), tau)
        np.testing.assert_allclose(Q, g[f"Q_case{c}"], rtol=0, atol=1e-14)


def test_barrier_known_answer(K):
    sig = np.zeros((1, 1, 2, 2)); sig[0, 0, 0, 1] = sig[0, 0, 1, 0] = 1e9
    cat = np.zeros((1, 1, 1, 2, 2)); cat[0, 0, 0, 0, 1] = cat[0, 0, 0, 1, 0] = 0.1
    Q = np.zeros((1, 1, 1))
    K.compute_barrier_2d(Q, np.ones((1, 1, 1)), sig, cat, 1.0, np.zeros((1, 1, 2)), np.full((1, 1), -np.inf), 0.0,
                         np.zeros((1, 1, 2, 2)), 2.0, 0, np.inf)
    assert abs(Q[0, 0, 0] - (1.0 - 0.6241509)) < 1e-12


def test_rates_golden(K, golden):
    g = golden("kmc2d_16x12")
    for T in (300.0, 0.0):
        for cm in (False, True):
            tag = f"T{int(T)}_c{int(cm)}"
            r, idx, total = K.compute_rates_2d(g["Q_rates"], 1.0, T, 1e13, cascade_mode=cm)
            np.testing.assert_array_equal(idx, g[f"indices_{tag}"])
            np.testing.assert_allclose(r, g[f"rates_{tag}"], rtol=1e-15, atol=0)
            assert total == np.add.accumulate(r)[-1]  # the sequential chain, bit for bit


def test_select_golden_bit_exact(K, golden):
    g = golden("kmc2d_16x12")
    rates, total = g["rates_T300_c0"], float(g["total_T300_c0"])
    for u, k in zip(g["sel_u"], g["sel_idx"]):
        assert K.select_event_2d_u(rates, total, u) == k


def test_flip_golden_bit_exact(K, golden):
    g = golden("kmc2d_16x12")
    ep, sp, tl = g["flip_in_eps_p"].copy(), g["flip_in_soft"].copy(), g["flip_in_tlast"].copy()
    for (x, y, m, t, jp, jt, gmax, jn) in g["flips"]:
        K.apply_flip_soa_2d(ep, sp, tl, g["catalog"], int(x), int(y), int(m), t, jp, jt, gmax, jn)
    np.testing.assert_array_equal(ep, g["flip_out_eps_p"])
    np.testing.assert_array_equal(sp, g["flip_out_soft"])
    np.testing.assert_array_equal(tl, g["flip_out_tlast"])


def test_full_size_barrier_rates_select(K):
    # 256^2 x 8 modes (524288 events), seeded state
    rng = np.random.default_rng(1)
    nx = ny = 256; M = 8
    cat, Q0 = W.kmc2d_state(nx, ny, M, rng)
    sig = 2e9 * rng.standard_normal((nx, ny, 2, 2))
    soft = np.zeros((nx, ny, 2)); tl = np.full((nx, ny), -np.inf); prev = np.zeros((nx, ny, 2, 2))
    Q = np.zeros((nx, ny, M)); Qo = np.zeros((nx, ny, M))
    K.compute_barrier_2d(Q, Q0, sig, cat, 1.0, soft, tl, 0.0, prev, 2.0, 0, np.inf)
    OK.compute_barrier(Qo, Q0, sig, cat, 1.0, soft, tl, 0.0, prev, 2.0, 0, np.inf)
    np.testing.assert_allclose(Q, Qo, rtol=0, atol=1e-13)
    r, idx, total = K.compute_rates_2d(Q, 1.0, 300.0, 1e13, cascade_mode=False)
    ro, _, _ = OK.compute_rates(Q, 1.0, 300.0, 1e13, cascade_mode=False)
    np.testing.assert_allclose(r, ro, rtol=1e-14, atol=0)
    S = np.add.accumulate(r)
    assert total == S[-1]
    draws = list(rng.random(40)) + [0.0, np.nextafter(1.0, 0.0)]
    # draws that land exactly on partial sums
    for k in (0, 1, 1000, 262143, len(r) - 2):
        draws.append(S[k] / total)
    for u in draws:
        if not (0.0 <= u < 1.0):
            continue
        assert K.select_event_2d_u(r, total, u) == OK.select_event(r, total, u)


def test_select_edges(K):
    assert K.select_event_2d_u(np.zeros(5), 0.0, 0.3) == -1
    r = np.array([0.0, 0.0, 1.0, 0.0])
    assert K.select_event_2d_u(r, 1.0, 0.0) == OK.select_event_loop(r, 1.0, 0.0) == 0
    assert K.select_event_2d_u(r, 1.0, 0.999) == OK.select_event_loop(r, 1.0, 0.999) == 2
    # total larger than the sum: falls off the end -> len-1
    assert K.select_event_2d_u(r, 2.0, 0.9) == OK.select_event_loop(r, 2.0, 0.9) == 3


def test_kmc3d_golden():
    from mgkmc_b200 import stz as S
    from tests.conftest import load_golden
    g = load_golden("kmc3d_6x5x4")
    Q = np.zeros_like(g["Q0"])
    S.compute_barrier(Q, g["Q0"], g["sig"], g["catalog"], 1.0, g["soft_prop"], g["last_event_time"], 1e-3,
                      g["prev_dir"], 0.5, 1, 5e-4)
    np.testing.assert_allclose(Q, g["Q"], rtol=0, atol=1e-14)
    Q2 = np.zeros_like(g["Q0"])
    S.compute_barrier(Q2, g["Q0"], g["sig"], g["catalog"], 1.0, g["soft_prop"], g["last_event_time"], 1e-3,
                      g["prev_dir"], 0.5, 0, np.inf)
    np.testing.assert_allclose(Q2, g["Q_iso"], rtol=0, atol=1e-14)
    r, idx, total = S.compute_rates(g["Q"], 1.0, 300.0, 1e13, cascade_mode=False)
    np.testing.assert_array_equal(idx, g["indices"])
    np.testing.assert_allclose(r, g["rates"], rtol=1e-15, atol=0)
    for u, k in zip(g["sel_u"], g["sel_idx"]):
        assert S.select_event_u(g["rates"], float(g["total"]), u) == k
    ep, sp, tl = g["flip_in_eps_p"].copy(), g["flip_in_soft"].copy(), g["flip_in_tlast"].copy()
    for (x, y, z, m, t, jp, jt, gmax, jn) in g["flips"]:
        S.apply_flip_soa(ep, None, sp, tl, g["catalog"], int(x), int(y), int(z), int(m), t, jp, jt, gmax, jn)
    np.testing.assert_array_equal(ep, g["flip_out_eps_p"])
    np.testing.assert_array_equal(sp, g["flip_out_soft"])
    np.testing.assert_array_equal(tl, g["flip_out_tlast"])


def _prefix_gpu(rates):
    import torch
    from mgkmc_b200 import _lib as L
    n = rates.size
    tr = torch.from_numpy(np.ascontiguousarray(rates, dtype=np.float64)).cuda()
    prefix = torch.full((max(n, 1),), np.nan, dtype=torch.float64, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    tot = torch.zeros(1, dtype=torch.float64, device="cuda")
    L.check(L.lib().mgk_kmc_prefix(L.ptr(tr), n, L.ptr(prefix), L.ptr(cnt), L.ptr(tot), L.stream_ptr()),
            "mgk_kmc_prefix")
    return prefix.cpu().numpy()[:n], float(tot.item())


def _tie_at(r, j, k=3):
    # make r[j] land exactly halfway between two doubles of the running sum
    # before it (a tie: its rounding depends on the parity of that sum)
    s = np.cumsum(r[:j])[-1]
    r[j] = (k + 0.5) * np.spacing(s)


@pytest.mark.parametrize("case", ["kmc", "wild", "zeros_subnormal_huge", "ties", "all_ties", "empty", "one",
                                  "large", "late_ties", "jump", "n8192", "n8193", "n8195", "n8196", "n16387"])
def test_exact_prefix_bit_for_bit(case):
    # the parallel exact running sum against the sequential loop (np.cumsum
    # adds left to right): every partial sum and the total, bit for bit
    rng = np.random.default_rng(7)
    if case == "kmc":
        r = 1e13 * np.exp(-rng.normal(1.0, 0.15, 200_000) / 0.02585)
    elif case == "wild":
        r = np.exp(rng.uniform(-700, 700, 50_000))
    elif case == "zeros_subnormal_huge":
        r = rng.random(30_000)
        r[::7] = 0.0
        r[5] = 5e-324
        r[1000] = 1e300
    elif case == "ties":  # halfway cases whose rounding depends on the parity of the sum
        r = np.full(40_000, 2.0 ** -53)
        r[0] = 1.0
        r[1::3] = 3 * 2.0 ** -53
    elif case == "all_ties":
        r = np.full(20_000, 1.5 * 2.0 ** -52)
        r[0] = 1.0
    elif case == "empty":
        r = np.zeros(0)
    elif case == "one":
        r = np.array([0.37])
    elif case == "late_ties":  # ties deep inside later chunks of an otherwise regular array
        r = 1e13 * np.exp(-rng.normal(1.0, 0.15, 200_000) / 0.02585)
        for j in (9_000, 100_000, 150_007, 199_999):
            _tie_at(r, j)
    elif case == "jump":  # a rate that moves the sum up many binades in the middle of a chunk
        r = rng.random(100_000)
        r[50_000] = 1e6
        r[70_003] = 1e12
    elif case.startswith("n"):  # chunk boundaries: last chunk of 0, 1, 3, 4 and 3 rates
        r = 1e13 * np.exp(-rng.normal(1.0, 0.15, int(case[1:])) / 0.02585)
    else:
        r = 1e13 * np.exp(-rng.normal(1.0, 0.15, 8_388_608) / 0.02585)  # 1024^2 x 8 modes
    p, tot = _prefix_gpu(r)
    ref = np.cumsum(r)
    assert np.array_equal(p.view(np.int64), ref.view(np.int64))
    assert tot == (ref[-1] if r.size else 0.0)


@pytest.mark.parametrize("n,T", [(64, 300.0), (256, 300.0), (96, 0.0)])
def test_fused_barrier_total(n, T):
    # the fused barrier + rate + block-sum pass of the fast selection mode:
    # barriers bit-equal to the barrier kernel's, the total equal to the sum
    # of the two-pass rates up to FP64 summation order
    import torch
    from mgkmc_b200 import _lib as L
    rng = np.random.default_rng(3)
    cat, Q0 = W.kmc2d_state(n, n, 8, rng)
    sig = 1e8 * rng.standard_normal((n, n, 2, 2))
    soft = np.abs(0.1 * rng.standard_normal((n, n, 2)))
    tl = rng.uniform(-1e-9, 0.0, (n, n))
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()
    tQ0, tsig, tcat, tsoft, ttl = d(Q0), d(sig), d(cat), d(soft), d(tl)
    Qa, Qb = torch.zeros_like(tQ0), torch.zeros_like(tQ0)
    lib, S = L.lib(), L.stream_ptr()
    tau = 1e-10
    L.check(lib.mgk_kmc2d_barrier(n, n, 8, L.ptr(Qa), L.ptr(tQ0), L.ptr(tsig), L.ptr(tcat), 1.0, L.ptr(tsoft),
                                  L.ptr(ttl), 0.0, None, 2.0, 0, tau, S), "barrier")
    nm = n * n * 8
    work = torch.empty(int(lib.mgk_kmc_scan_work_bytes(nm)), dtype=torch.uint8, device="cuda")
    tot = torch.zeros(1, dtype=torch.float64, device="cuda")
    L.check(lib.mgk_kmc2d_barrier_total(n, n, 8, L.ptr(Qb), L.ptr(tQ0), L.ptr(tsig), L.ptr(tcat), 1.0, L.ptr(tsoft),
                                        L.ptr(ttl), 0.0, None, 2.0, 0, tau, 1.0, None, T, 1e13, L.ptr(tot),
                                        L.ptr(work), S), "barrier_total")
    assert torch.equal(Qa, Qb)
    rates = torch.empty(nm, dtype=torch.float64, device="cuda")
    L.check(lib.mgk_kmc2d_rates_only(n, n, 8, L.ptr(Qa), 1.0, None, T, 1e13, L.ptr(rates), S), "rates_only")
    r = rates.cpu().numpy()
    assert abs(float(tot.item()) - np.sum(r)) <= 1e-13 * np.sum(r)


@pytest.mark.parametrize("nx,ny,M,R,x,y,m", [(24, 20, 4, 3, 1, 18, 2), (5, 4, 3, 3, 4, 1, 1), (16, 16, 8, 0, 7, 0, 5)])
def test_patch_bit_exact(nx, ny, M, R, x, y, m):
    # fast-patching stress update (kmc_simulator.py:1052-1069) against the
    # oracle's numpy form, bit for bit: with the unit macro-strain term, through
    # the compacted index list, a window that wraps (5 x 4 grid, R = 3), R = 0
    import torch
    from mgkmc_b200 import _lib as L
    from oracle import kmc_driver as OD
    rng = np.random.default_rng(nx * 100 + R)
    W_ = 2 * R + 1
    sig0 = rng.normal(0, 1e8, (nx, ny, 2, 2))
    unit = rng.normal(0, 5e10, (nx, ny, 2, 2))
    kern = rng.normal(0, 1e10, (2, W_, W_, 2, 2))
    miss = rng.normal(0, 1e6, (2, 2, 2))
    cat = rng.normal(0, 0.05, (nx, ny, M, 2, 2))
    scale = 3.7e-7
    flat = (x * ny + y) * M + m
    dev = torch.device("cuda")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    tsig, tunit, tkern, tmiss, tcat = t(sig0), t(unit), t(kern), t(miss), t(cat)
    indices = t(np.array([5, flat, 2], dtype=np.int64))
    sel = t(np.array([1], dtype=np.int64))
    lib, S = L.lib(), L.stream_ptr()
    L.check(lib.mgk_kmc2d_patch(nx, ny, M, L.ptr(tsig), L.ptr(tunit), scale, L.ptr(tkern), L.ptr(tmiss), R,
                                L.ptr(tcat), L.ptr(sel), L.ptr(indices), S), "patch")
    ref = sig0.copy()
    OD.apply_patch_2d(ref, x, y, cat[x, y, m, 0, 0], cat[x, y, m, 0, 1], kern, miss, unit=unit, scale=scale)
    np.testing.assert_array_equal(tsig.cpu().numpy(), ref)
    # a negative selection leaves the patch out; no selection: only the unit term
    neg = t(np.array([-1], dtype=np.int64))
    tsig2 = t(sig0)
    L.check(lib.mgk_kmc2d_patch(nx, ny, M, L.ptr(tsig2), None, 0.0, L.ptr(tkern), L.ptr(tmiss), R, L.ptr(tcat),
                                L.ptr(neg), None, S), "patch")
    np.testing.assert_array_equal(tsig2.cpu().numpy(), sig0)
    L.check(lib.mgk_kmc2d_patch(nx, ny, M, L.ptr(tsig2), L.ptr(tunit), scale, None, None, R, None, None, None, S),
            "patch")
    np.testing.assert_array_equal(tsig2.cpu().numpy(), sig0 + unit * scale)


@pytest.mark.parametrize("nx,ny,R", [(24, 20, 3), (14, 12, 7)])
def test_patch_setup(nx, ny, R):
    # windows and missing means of kmc_simulator.py:229-261 from given responses
    import torch
    from mgkmc_b200 import _lib as L
    rng = np.random.default_rng(R)
    r = rng.normal(0, 1e9, (2, nx, ny, 2, 2))
    dev = torch.device("cuda")
    tr = torch.from_numpy(r).to(dev)
    kern = torch.empty((2, 2 * R + 1, 2 * R + 1, 2, 2), dtype=torch.float64, device=dev)
    miss = torch.empty((2, 2, 2), dtype=torch.float64, device=dev)
    L.check(L.lib().mgk_kmc2d_patch_setup(nx, ny, R, L.ptr(tr[0]), L.ptr(tr[1]), L.ptr(kern), L.ptr(miss),
                                          L.stream_ptr()), "patch_setup")
    ix = (np.arange(-R, R + 1) + nx // 2) % nx
    iy = (np.arange(-R, R + 1) + ny // 2) % ny
    for b in range(2):
        crop = r[b][ix[:, None], iy[None, :]]
        np.testing.assert_array_equal(kern[b].cpu().numpy(), crop)
        want = np.mean(r[b], axis=(0, 1)) - np.sum(crop, axis=(0, 1)) / (nx * ny)
        np.testing.assert_allclose(miss[b].cpu().numpy(), want, rtol=0, atol=1e-12 * np.max(np.abs(r)))
