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


class _Fake3D:
    """A stand-in for Kmc3D's checkpoint surface (no device needed)."""

    def __init__(self, rng):
        self.nx, self.ny, self.nz, self.M = 4, 3, 2, 2
        sh = (4, 3, 2)
        self.p = dict(T=300.0, gamma0=0.1, nu0=1e13, strain_rate=1e7, jp=0.0, jt=0.0, jn=0.0, cap=2.0)
        self.selection, self.ls_start = "fast", "warm"
        self.ls = type("P", (), {"precision": "mixed"})()
        self._st = {"E": rng.random(sh), "nu": rng.random(sh), "eps": rng.random(sh + (3, 3)),
                    "sig": rng.random(sh + (3, 3)), "eps_p": rng.random(sh + (3, 3)), "soft": rng.random(sh + (4,)),
                    "Q": rng.random(sh + (2,)), "Q0": rng.random(sh + (2,)), "catalog": rng.random(sh + (2, 3, 3)),
                    "t_last": rng.random(sh), "prev": rng.random(sh + (3, 3)), "eps_macro": rng.random((3, 3)),
                    "time": 1.25e-9, "events": [(1, 2, 0, 1, 3.0e-10), (3, 0, 1, 0, 9.5e-10)], "n_solves": 17,
                    "steps_done": 5}

    def state_dict(self):
        return dict(self._st)


def test_trajectory_roundtrip_3d(tmp_path):
    # the 3D trajectory checkpoint: the reference's aqs.py layout (flips as
    # (x, y, z, m)) plus the resume group, read back into a state dict
    rng = np.random.default_rng(2)
    sim = _Fake3D(rng)
    g = np.random.default_rng(99)
    g.random(3)
    path = C.save_trajectory(str(tmp_path / "t3"), sim, g, fmt="npz")
    data, attrs = C.load(path)
    assert data["history/flips"].shape == (2, 4) and attrs["metadata"]["nz"] == 2
    st, rng2, meta = C.load_trajectory(path)
    for k in ("eps", "sig", "eps_p", "soft", "Q", "Q0", "catalog", "t_last", "prev", "eps_macro", "E", "nu"):
        np.testing.assert_array_equal(st[k], sim._st[k])
    assert st["events"] == sim._st["events"] and st["steps_done"] == 5 and st["n_solves"] == 17
    np.testing.assert_array_equal(rng2.random(4), g.random(4))


def test_trajectory_without_events(tmp_path):
    # a checkpoint taken before the first event: an empty flip history that
    # still reads back as (0, 4) and an empty event list
    sim = _Fake3D(np.random.default_rng(4))
    sim._st["events"] = []
    path = C.save_trajectory(str(tmp_path / "t0"), sim, np.random.default_rng(1), fmt="npz")
    data, _ = C.load(path)
    assert data["history/flips"].shape == (0, 4)
    st, _, _ = C.load_trajectory(path)
    assert st["events"] == []


class _Fake2D:
    """A stand-in for Kmc2D's checkpoint surface (no device needed)."""

    def __init__(self, rng):
        self.nx, self.ny, self.M = 6, 4, 3
        sh = (6, 4)
        self.p = dict(T=250.0, gamma0=0.1, nu0=1e13, strain_rate=1e7, jp=0.1, jt=0.2, jn=0.3, cap=2.0)
        self.selection, self.ls_start = "exact", "cold"
        self.ls = type("P", (), {"precision": "fp64"})()
        self.stability_threshold = -0.05
        self._st = {"E": rng.random(sh), "nu": rng.random(sh), "eps": rng.random(sh + (2, 2)),
                    "sig": rng.random(sh + (2, 2)), "eps_p": rng.random(sh + (2, 2)), "soft": rng.random(sh + (2,)),
                    "Q": rng.random(sh + (3,)), "Q0": rng.random(sh + (3,)), "catalog": rng.random(sh + (3, 2, 2)),
                    "t_last": rng.random(sh), "prev": rng.random(sh + (2, 2)), "eps_macro": rng.random((2, 2)),
                    "time": 3.5e-9, "events": [(5, 1, 2, 1.0e-9), (0, 3, 0, 2.5e-9), (2, 2, 1, 3.0e-9)],
                    "n_solves": 9, "steps_done": 4, "unit_ready": True, "flips_since_sync": 2}

    def state_dict(self):
        return dict(self._st)


def test_trajectory_roundtrip_2d(tmp_path):
    # the 2D trajectory checkpoint: flips as (x, y, m), nz = 1 in the
    # metadata, the fast-patching counters and the cascade threshold kept
    sim = _Fake2D(np.random.default_rng(6))
    g = np.random.default_rng(7)
    g.normal(size=5)
    path = C.save_trajectory(str(tmp_path / "t2"), sim, g, fmt="npz")
    data, attrs = C.load(path)
    assert data["history/flips"].shape == (3, 3) and data["history/flips"].dtype == np.int32
    meta = attrs["metadata"]
    assert meta["nz"] == 1 and meta["M"] == 3 and meta["stability_threshold"] == -0.05
    assert meta["temperature"] == 250.0 and meta["neighbor_softening_fraction"] == 0.3
    np.testing.assert_array_equal(data["fields/Tlocal"], np.full((6, 4), 250.0))
    st, g2, _ = C.load_trajectory(path)
    for k in ("eps", "sig", "eps_p", "soft", "Q", "Q0", "catalog", "t_last", "prev", "eps_macro", "E", "nu"):
        np.testing.assert_array_equal(st[k], sim._st[k])
    assert st["events"] == sim._st["events"] and st["unit_ready"] is True and st["flips_since_sync"] == 2
    assert st["time"] == 3.5e-9 and st["steps_done"] == 4 and st["n_solves"] == 9
    np.testing.assert_array_equal(g2.normal(size=4), g.normal(size=4))
