"""Host-side parts of the serving layer: the request stream and footprints."""
import numpy as np

from mgkmc_b200.serving import SIZES_2D, SIZES_3D, Request, footprint_bytes, request_stream


def test_stream_statistics():
    reqs = request_stream(rate=200.0, duration=60.0, seed=3)
    n = len(reqs)
    assert 11000 < n < 13000  # Poisson(12000)
    t = np.array([r.t_arrival for r in reqs])
    assert np.all(np.diff(t) > 0) and t[-1] <= 60.0
    assert abs(np.mean(np.diff(t)) - 1 / 200.0) < 2e-4
    assert abs(np.mean([r.kind == "trajectory" for r in reqs]) - 0.4) < 0.02
    assert abs(np.mean([r.dim == 3 for r in reqs]) - 0.3) < 0.02
    assert {r.n for r in reqs if r.dim == 2} == set(SIZES_2D)
    assert {r.n for r in reqs if r.dim == 3} == set(SIZES_3D)
    assert request_stream(seed=3)[:50] == reqs[:50]  # reproducible


def test_footprints_grow_with_size():
    a = footprint_bytes(Request(0, 0, "solve", 2, 256, 0))
    b = footprint_bytes(Request(0, 0, "trajectory", 2, 256, 0))
    c = footprint_bytes(Request(0, 0, "solve", 3, 64, 0))
    assert 0 < a < b and c > a
    assert footprint_bytes(Request(0, 0, "solve", 2, 512, 0)) == 4 * a
