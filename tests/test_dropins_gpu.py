"""The per-event numpy drop-ins (kmc_simulator_functions) on the benchmark's
256^2 x 8 state: the flip moves only its neighbourhood and equals the
oracle's bit for bit; selection on the rates of compute_rates_2d reuses their
device running sums and picks the same index as a fresh upload; barriers with
device mirrors equal barriers from full uploads over a run of flips and host
redraws."""
import time

import numpy as np
import pytest

from mgkmc_b200 import workloads as W
from oracle import kmc as OK

pytestmark = pytest.mark.gpu


def _state(n=256, M=8, seed=1):
    rng = np.random.default_rng(seed)
    cat, Q0 = W.kmc2d_state(n, n, M, rng)
    eps_p = 0.01 * rng.standard_normal((n, n, 2, 2))
    soft = np.abs(0.1 * rng.standard_normal((n, n, 2)))
    tl = np.where(rng.random((n, n)) < 0.5, -np.inf, rng.uniform(0, 1e-9, (n, n)))
    return rng, cat, Q0, eps_p, soft, tl


@pytest.mark.parametrize("jn,x,y", [(0.0, 17, 200), (0.2, 0, 255), (0.2, 128, 3)])
def test_flip_matches_oracle_and_moves_only_the_neighbourhood(jn, x, y):
    from mgkmc_b200 import kmc_simulator_functions as K
    rng, cat, Q0, eps_p, soft, tl = _state()
    a = (eps_p.copy(), soft.copy(), tl.copy())
    b = (eps_p.copy(), soft.copy(), tl.copy())
    K.apply_flip_soa_2d(*a, cat, x, y, 5, 2e-9, 10.0, 30.0, 2.0, jn)  # warm-up (plans, context)
    a = (eps_p.copy(), soft.copy(), tl.copy())
    t0 = time.perf_counter()
    K.apply_flip_soa_2d(*a, cat, x, y, 5, 2e-9, 10.0, 30.0, 2.0, jn)
    dt = time.perf_counter() - t0
    OK.apply_flip_2d(*b, cat, x, y, 5, 2e-9, 10.0, 30.0, 2.0, jn)
    for u, v in zip(a, b):
        np.testing.assert_array_equal(u, v)
    print(f"apply_flip_soa_2d at 256^2 x 8, jn={jn}: {1e3 * dt:.3f} ms")
    assert dt < 0.05


def test_selection_reuses_device_running_sums():
    from mgkmc_b200 import kmc_simulator_functions as K
    rng, cat, Q0, eps_p, soft, tl = _state()
    sig = 1e9 * rng.standard_normal((256, 256, 2, 2))
    Q = np.zeros_like(Q0)
    K.compute_barrier_2d(Q, Q0, sig, cat, 1.0, soft, tl, 0.0, np.zeros_like(eps_p), 2.0, 0, np.inf)
    rates, idx, total = K.compute_rates_2d(Q, 1.0, 300.0, 1e13, cascade_mode=False)
    assert not rates.flags.writeable
    for u in (0.0, 0.3, 0.77, np.nextafter(1.0, 0.0)):
        k1 = K.select_event_2d_u(rates, total, u)
        k2 = K.select_event_2d_u(np.array(rates), total, u)
        assert k1 == k2 == OK.select_event(np.array(rates), total, u)


def test_barrier_mirrors_follow_flips_and_redraws():
    from mgkmc_b200 import kmc_simulator_functions as K
    rng, cat, Q0, eps_p, soft, tl = _state(n=64)
    prev = np.zeros_like(eps_p)
    sig = 1e9 * rng.standard_normal((64, 64, 2, 2))
    Qa, Qb = np.zeros_like(Q0), np.zeros_like(Q0)
    try:
        for step in range(6):
            K.use_device_mirrors(True)
            K.compute_barrier_2d(Qa, Q0, sig, cat, 1.0, soft, tl, 1e-9 * step, prev, 2.0, 1, 1e-9)
            K.use_device_mirrors(False)
            K.compute_barrier_2d(Qb, Q0, sig, cat, 1.0, soft, tl, 1e-9 * step, prev, 2.0, 1, 1e-9)
            np.testing.assert_array_equal(Qa, Qb)
            K.use_device_mirrors(True)
            x, y, m = int(rng.integers(64)), int(rng.integers(64)), int(rng.integers(8))
            C = cat[x, y, m].copy()
            K.apply_flip_soa_2d(eps_p, soft, tl, cat, x, y, m, 1e-9 * step, 10.0, 30.0, 2.0, 0.2)
            prev[x, y] = C  # the driver's redraws of the flipped voxel (kmc_simulator.py:1030-1042)
            cat[x, y] = W.kmc2d_state(1, 1, 8, rng)[0][0, 0]
            Q0[x, y] = 0.3 + rng.random(8)
            sig = sig + 1e7 * rng.standard_normal(sig.shape)
    finally:
        K.use_device_mirrors(False)
