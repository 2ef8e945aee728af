"""VTK output: the node displacement against the reference's reconstruction
(golden), and a written file read back (mesh, connectivity, named arrays)."""
import numpy as np

from mgkmc_b200 import vtk as V


def test_displacement_matches_reference(golden):
    g = golden("vtk_displacement")
    assert np.max(np.abs(V.reconstruct_displacement(g["eps2"], 1.5) - g["u2"])) <= 1e-15
    assert np.max(np.abs(V.reconstruct_displacement(g["eps3"], 0.5) - g["u3"])) <= 1e-15


def test_export_round_trip(tmp_path):
    rng = np.random.default_rng(3)
    nx, ny = 5, 4
    eps = rng.normal(0, 0.01, (nx, ny, 2, 2))
    sig = rng.normal(0, 1e8, (nx, ny, 2, 2))
    ep = rng.normal(0, 0.01, (nx, ny, 2, 2))
    E, nu = rng.uniform(80e9, 100e9, (nx, ny)), rng.uniform(0.3, 0.4, (nx, ny))
    soft = rng.random((nx, ny, 2))
    f = V.export_to_vtk(str(tmp_path / "a.vtu"), eps, sig, E, nu, pixel=2.0, eps_plastic_field=ep,
                        soft_prop_field=soft, Tlocal=np.full((nx, ny), 300.0))
    pts, conn, pd, cd = V.read_vtu(f)
    assert pts.shape == ((nx + 1) * (ny + 1) * 2, 3) and conn.shape == (nx * ny, 8)
    assert np.allclose(pts[conn[0]], [[0, 0, 0], [0, 0, 2], [0, 2, 2], [0, 2, 0],
                                      [2, 0, 0], [2, 0, 2], [2, 2, 2], [2, 2, 0]])
    assert np.array_equal(cd["E"], E.ravel()) and np.array_equal(cd["sig_xy"], sig[..., 0, 1].ravel())
    assert np.array_equal(cd["eps_elastic_xx"], (eps - ep)[..., 0, 0].ravel())
    assert np.allclose(cd["eps_zz"], 0) and np.array_equal(cd["g_t"], soft[..., 1].ravel())
    tr = sig[..., 0, 0] + sig[..., 1, 1]
    s3 = np.zeros((nx, ny, 3, 3))
    s3[..., :2, :2] = sig
    s3 -= np.eye(3) * (tr / 3)[..., None, None]
    assert np.allclose(cd["sig_vm"], np.sqrt(1.5 * np.sum(s3 ** 2, axis=(-2, -1))).ravel(), rtol=1e-14)
    assert np.array_equal(pd["displacement"], V.reconstruct_displacement(eps, 2.0).reshape(-1, 3))
    assert {"temperature", "eps_plastic_vm", "eps_vm", "eps_elastic_vm"} <= set(cd)
