"""Checkpoint containers on CPU: the reference's group / dataset / attribute
layout (mgkmc/linear_elastic_simulator.py:568-607, mgkmc/aqs.py:1207-1267)
written and read back, and the trajectory resume record."""
import numpy as np

from mgkmc_b200 import checkpoint as C


def test_roundtrip_2d_layout(tmp_path):
    rng = np.random.default_rng(0)
    E, nu = rng.random((8, 6)), rng.random((8, 6))
    eps, sig = rng.random((8, 6, 2, 2)), rng.random((8, 6, 2, 2))
    p = C.save_checkpoint_2d(str(tmp_path / "chk_000002"), 2, E, nu, eps, sig, eps.mean((0, 1)), sig.mean((0, 1)),
                             1.5, fmt="npz")
    data, attrs = C.load(p)
    assert set(data) == {"fields/eps_field", "fields/sig_field", "fields/E_field", "fields/nu_field",
                         "macro/eps_macro", "macro/sig_macro"}
    np.testing.assert_array_equal(data["fields/eps_field"], eps)
    np.testing.assert_array_equal(data["fields/nu_field"], nu)
    assert attrs["metadata"] == {"nx": 8, "ny": 6, "pixel": 1.5, "step": 2}


def test_roundtrip_3d_layout(tmp_path):
    rng = np.random.default_rng(1)
    E = rng.random((4, 6, 8))
    eps = rng.random((4, 6, 8, 3, 3))
    p = C.save_checkpoint_3d(str(tmp_path / "c3"), 7, E, E, eps, eps, eps.mean((0, 1, 2)), eps.mean((0, 1, 2)), 1.0,
                             fmt="npz")
    data, attrs = C.load(p)
    np.testing.assert_array_equal(data["fields/sig_field"], eps)
    assert attrs["metadata"]["nz"] == 8 and attrs["metadata"]["step"] == 7


def test_rng_state_roundtrip():
    g = np.random.default_rng(123)
    g.random(17)
    h = C._rng_from_json(C._rng_state_json(g))
    np.testing.assert_array_equal(g.random(5), h.random(5))
    np.testing.assert_array_equal(g.normal(size=3), h.normal(size=3))
