"""VTK output of voxel fields, in the layout of the reference's writer.

The reference writes its results with meshio (mgkmc/analysis/vtk.py:118-372
``export_to_vtk``): an unstructured grid of hexahedra, one per voxel, with
the voxel-centred fields as cell data and a displacement reconstructed from
the strain as point data.  meshio is not a dependency here, so the same mesh
and the same named arrays are written directly as a VTK XML unstructured
grid (``.vtu``: little-endian, UInt64 headers, base64-encoded raw arrays),
which ParaView and VTK read as they read the reference's files.
"""
import base64
import struct

import numpy as np

VTK_HEXAHEDRON = 12


def reconstruct_displacement(eps, pixel=1.0):
    """Node displacements (nx+1, ny+1, nz+1, 3) from a voxel strain field
    (mgkmc/analysis/vtk.py:4-116 reconstruct_displacement_element_centered):
    normal strains integrated along their axis from the first node, each
    engineering shear adding half of its voxel's value to the next node along
    the other axis, then the mean displacement of the x = 0 nodes removed.
    eps: (nx, ny, 2, 2) (a one-voxel-thick 3D field) or (nx, ny, nz, 3, 3)."""
    eps = np.asarray(eps, dtype=np.float64)
    if eps.ndim == 4:
        e3 = np.zeros(eps.shape[:2] + (1, 3, 3))
        e3[:, :, 0, :2, :2] = eps
        eps = e3
    nx, ny, nz = eps.shape[:3]
    ix = np.minimum(np.arange(nx + 1), nx - 1)
    jy = np.minimum(np.arange(ny + 1), ny - 1)
    kz = np.minimum(np.arange(nz + 1), nz - 1)
    u = np.zeros((nx + 1, ny + 1, nz + 1, 3))
    # normal strains: running sums along the axis, from zero at the first node
    u[1:, :, :, 0] = np.cumsum(eps[:, jy][:, :, kz][..., 0, 0] * pixel, axis=0)
    u[:, 1:, :, 1] = np.cumsum(eps[ix][:, :, kz][..., 1, 1] * pixel, axis=1)
    u[:, :, 1:, 2] = np.cumsum(eps[ix][:, jy][..., 2, 2] * pixel, axis=2)
    gxy, gxz, gyz = eps[..., 0, 1], eps[..., 0, 2], eps[..., 1, 2]
    # shears: half of the neighbouring voxel's tensorial shear, node by node
    u[:, 1:, :, 0] += 0.5 * gxy[ix][:, :, kz] * pixel
    u[:, :, 1:, 0] += 0.5 * gxz[ix][:, jy] * pixel
    u[1:, :, :, 1] += 0.5 * gxy[:, jy][:, :, kz] * pixel
    u[:, :, 1:, 1] += 0.5 * gyz[ix][:, jy] * pixel
    u[1:, :, :, 2] += 0.5 * gxz[:, jy][:, :, kz] * pixel
    u[:, 1:, :, 2] += 0.5 * gyz[ix][:, :, kz] * pixel
    u -= u[0].mean(axis=(0, 1)).reshape(1, 1, 1, 3)
    return u


def _vm_dev(t, scale):
    tr = np.trace(t, axis1=-2, axis2=-1)[..., None, None]
    dev = t - np.eye(3) * tr / 3
    return np.sqrt(scale * np.sum(dev ** 2, axis=(-2, -1)))


def _as3d(a, nx, ny):
    if a.ndim == 4:
        out = np.zeros((nx, ny, 1, 3, 3))
        out[:, :, 0, :a.shape[-2], :a.shape[-1]] = a
        return out
    return a


def _b64(arr):
    raw = np.ascontiguousarray(arr).tobytes()
    return base64.b64encode(struct.pack("<Q", len(raw)) + raw).decode("ascii")


def _data_array(name, arr, ncomp=1, vtype="Float64"):
    attrs = f' type="{vtype}"' + (f' Name="{name}"' if name else "") + \
        (f' NumberOfComponents="{ncomp}"' if ncomp > 1 else "") + ' format="binary"'
    return f"<DataArray{attrs}>{_b64(arr)}</DataArray>"


def write_vtu(filename, points, hexes, point_data, cell_data):
    """A VTK XML unstructured grid of hexahedra: points (P, 3), hexes (C, 8)
    node indices, point_data / cell_data {name: (P or C,) or (P, 3) array}."""
    P, C = len(points), len(hexes)
    out = ['<?xml version="1.0"?>',
           '<VTKFile type="UnstructuredGrid" version="1.0" byte_order="LittleEndian" header_type="UInt64">',
           '<UnstructuredGrid>', f'<Piece NumberOfPoints="{P}" NumberOfCells="{C}">',
           '<Points>', _data_array("", np.asarray(points, "<f8"), 3), '</Points>',
           '<Cells>',
           _data_array("connectivity", np.asarray(hexes, "<i8").ravel(), 1, "Int64"),
           _data_array("offsets", 8 * np.arange(1, C + 1, dtype="<i8"), 1, "Int64"),
           _data_array("types", np.full(C, VTK_HEXAHEDRON, dtype=np.uint8), 1, "UInt8"),
           '</Cells>', '<PointData>']
    for k, v in point_data.items():
        v = np.asarray(v, "<f8")
        out.append(_data_array(k, v, v.shape[1] if v.ndim == 2 else 1))
    out.append('</PointData>')
    out.append('<CellData>')
    for k, v in cell_data.items():
        out.append(_data_array(k, np.asarray(v, "<f8").ravel()))
    out += ['</CellData>', '</Piece>', '</UnstructuredGrid>', '</VTKFile>']
    with open(filename, "w") as f:
        f.write("\n".join(out) + "\n")
    return filename


def read_vtu(filename):
    """(points, connectivity, point_data, cell_data) of a file written by
    write_vtu (for checks and round trips)."""
    import xml.etree.ElementTree as ET
    root = ET.parse(filename).getroot()
    dt = {"Float64": "<f8", "Int64": "<i8", "UInt8": "u1"}

    def arr(el):
        raw = base64.b64decode(el.text.strip())
        n = struct.unpack("<Q", raw[:8])[0]
        a = np.frombuffer(raw[8:8 + n], dtype=dt[el.get("type")])
        nc = int(el.get("NumberOfComponents", "1"))
        return a.reshape(-1, nc) if nc > 1 else a

    piece = root.find("UnstructuredGrid/Piece")
    points = arr(piece.find("Points/DataArray"))
    conn = {el.get("Name"): arr(el) for el in piece.find("Cells")}
    pd = {el.get("Name"): arr(el) for el in piece.find("PointData")}
    cd = {el.get("Name"): arr(el) for el in piece.find("CellData")}
    return points, conn["connectivity"].reshape(-1, 8), pd, cd


def export_to_vtk(filename, eps, sig, E, nu, pixel=1.0, grid=None, include_plastic=True,
                  match_matplotlib_orientation=False, eps_plastic_field=None, soft_prop_field=None, Tlocal=None):
    """mgkmc/analysis/vtk.py:118-372 export_to_vtk: voxel fields as hexahedral
    cells.  eps, sig: (nx, ny, 2, 2) or (nx, ny, nz, 3, 3); E, nu: voxel
    fields; cell data E, nu, the strain, elastic strain and stress
    components, von Mises stress and strains, [temperature], [plastic strain
    components and von Mises], [g_p, g_t of soft_prop_field]; point data the
    reconstructed displacement.  ``grid`` (the reference's legacy voxel
    objects) is not supported; ``match_matplotlib_orientation`` is accepted
    and, as in the reference, changes nothing."""
    if grid is not None:
        raise NotImplementedError("export_to_vtk: the legacy voxel-object grid is not supported")
    eps = np.asarray(eps, dtype=np.float64)
    sig = np.asarray(sig, dtype=np.float64)
    if eps.ndim == 4:
        nx, ny = eps.shape[:2]
        nz = 1
        E = np.asarray(E).reshape(nx, ny, 1)
        nu = np.asarray(nu).reshape(nx, ny, 1)
        eps, sig = _as3d(eps, nx, ny), _as3d(sig, nx, ny)
    else:
        nx, ny, nz = np.shape(E)
    ep = None
    if eps_plastic_field is not None:
        ep = np.asarray(eps_plastic_field, dtype=np.float64)
        ep = _as3d(ep, nx, ny) if ep.ndim == 4 else ep
    eel = eps - ep if ep is not None else eps
    x, y, z = (np.arange(n + 1) * pixel for n in (nx, ny, nz))
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    points = np.column_stack([X.ravel(), Y.ravel(), Z.ravel()])
    NYZ, NZ = (ny + 1) * (nz + 1), nz + 1
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    n0 = (i * NYZ + j * NZ + k).ravel()
    n2, n4 = n0 + NZ, n0 + NYZ
    hexes = np.stack([n0, n0 + 1, n2 + 1, n2, n4, n4 + 1, n4 + NZ + 1, n4 + NZ], axis=1)
    cd = {"E": E, "nu": nu}
    for pre, t in (("eps", eps), ("eps_elastic", eel), ("sig", sig)):
        for (a, b), lab in zip(((0, 0), (1, 1), (2, 2)), ("xx", "yy", "zz")):
            cd[f"{pre}_{lab}"] = t[..., a, b]
        for (a, b), lab in zip(((0, 1), (0, 2), (1, 2)), ("xy", "xz", "yz")):
            cd[f"{pre}_{lab}"] = t[..., a, b]
    order = ["E", "nu"] + [f"eps_{s}" for s in ("xx", "yy", "zz", "xy", "xz", "yz")] + \
        [f"eps_elastic_{s}" for s in ("xx", "yy", "zz", "xy", "xz", "yz")] + \
        [f"sig_{s}" for s in ("xx", "yy", "zz", "xy", "xz", "yz")]
    cell = {name: cd[name] for name in order}
    cell["sig_vm"] = _vm_dev(sig, 1.5)
    cell["eps_vm"] = _vm_dev(eps, 2.0 / 3.0)
    cell["eps_elastic_vm"] = _vm_dev(eel, 2.0 / 3.0)
    if Tlocal is not None:
        cell["temperature"] = np.asarray(Tlocal)
    if ep is not None:
        for (a, b), lab in zip(((0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)), ("xx", "yy", "zz", "xy", "xz", "yz")):
            cell[f"eps_plastic_{lab}"] = ep[..., a, b]
        cell["eps_plastic_vm"] = _vm_dev(ep, 2.0 / 3.0)
        if soft_prop_field is not None:
            sp = np.asarray(soft_prop_field)
            cell["g_p"], cell["g_t"] = sp[..., 0], sp[..., 1]
    u = reconstruct_displacement(eps, pixel)
    return write_vtu(filename, points, hexes, {"displacement": u.reshape(-1, 3)}, cell)
