"""Checkpoints of device-resident simulation state, in the reference's layout.

The reference writes HDF5 files with h5py:

* ``save_checkpoint_2d`` / ``save_checkpoint_3d``
  (mgkmc/linear_elastic_simulator.py:568-607): group ``metadata`` (attrs nx,
  ny[, nz], pixel, step), group ``fields`` (eps_field, sig_field, E_field,
  nu_field), group ``macro`` (eps_macro, sig_macro);
* ``ThermalSimulation.save_checkpoint`` (mgkmc/aqs.py:1207-1267): group
  ``metadata`` (grid, STZ and rate attributes), ``fields`` (eps_field,
  sig_field, E_field, nu_field, Tlocal), ``grid`` (eps_plastic, soft_prop, Q,
  Q0, catalog, last_event_time), ``state`` (eps_macro), ``history/flips``.

The same group / dataset / attribute names are written here.  When h5py is
importable the file is HDF5 (gzip datasets, as the reference writes them);
otherwise the container is a numpy ``.npz`` archive whose keys are the HDF5
paths (``"fields/eps_field"``) and whose attributes are 0-d entries under
``"<group>/@<name>"``.  ``load`` reads either.

A trajectory checkpoint (``save_trajectory`` / ``load_trajectory``) adds what
a bit-exact resume of the device-resident KMC driver needs beyond the
reference's layout, under the group ``resume``: the clock, the AQS steps
done, the event list, the solve count, the previous-direction field, the
numpy Generator state of the trajectory's draws and the per-voxel eigenstrain
the LS plan holds.  Checkpoints are taken between AQS steps, where the
reference takes them (kmc_simulator.py:796-1157 logs and checkpoints after an
elastic step).
"""
import datetime
import json
import os

import numpy as np

try:  # the reference's container format, when the library is present
    import h5py  # noqa: F401
    _HAVE_H5PY = True
except ImportError:
    _HAVE_H5PY = False


def _to_np(a):
    if hasattr(a, "detach"):
        return a.detach().cpu().numpy()
    return np.asarray(a)


def write(path, groups, attrs, fmt=None):
    """Writes ``groups`` ({"group/name": array}) and ``attrs``
    ({"group": {name: scalar or str}}).  ``fmt``: "h5", "npz" or None (h5 when
    h5py is importable).  Returns the path written."""
    fmt = fmt or ("h5" if _HAVE_H5PY else "npz")
    if fmt == "h5":
        import h5py
        if not path.endswith(".h5"):
            path += ".h5"
        # file locking off for the process, as the reference's writers set it
        # (linear_elastic_simulator.py:573, aqs.py:1209)
        os.environ["HDF5_USE_FILE_LOCKING"] = "FALSE"
        with h5py.File(path, "w") as f:
            for g, d in attrs.items():
                grp = f.require_group(g)
                for k, v in d.items():
                    grp.attrs[k] = v
            for k, v in groups.items():
                v = _to_np(v)
                # chunked (compressed) storage needs a non-empty array: an
                # empty event list is stored contiguous
                f.create_dataset(k, data=v, compression="gzip" if v.ndim >= 2 and v.size > 0 else None)
        return path
    if fmt != "npz":
        raise ValueError(f"unknown checkpoint format {fmt!r}")
    if not path.endswith(".npz"):
        path += ".npz"
    flat = {k: _to_np(v) for k, v in groups.items()}
    for g, d in attrs.items():
        for k, v in d.items():
            flat[f"{g}/@{k}"] = np.asarray(v)
    with open(path, "wb") as f:
        np.savez_compressed(f, **flat)
    return path


def load(path):
    """(datasets {"group/name": array}, attrs {"group": {name: value}})."""
    if path.endswith(".h5") or (not path.endswith(".npz") and os.path.exists(path + ".h5")):
        import h5py
        path = path if path.endswith(".h5") else path + ".h5"
        data, attrs = {}, {}
        with h5py.File(path, "r") as f:
            def visit(name, obj):
                if isinstance(obj, h5py.Dataset):
                    data[name] = obj[()]
                if obj.attrs:
                    attrs[name] = dict(obj.attrs)
            f.visititems(visit)
        return data, attrs
    path = path if path.endswith(".npz") else path + ".npz"
    data, attrs = {}, {}
    with np.load(path, allow_pickle=False) as z:
        for k in z.files:
            g, _, name = k.rpartition("/")
            if name.startswith("@"):
                v = z[k]
                attrs.setdefault(g, {})[name[1:]] = v.item() if v.ndim == 0 else v
            else:
                data[k] = z[k]
    return data, attrs


def save_checkpoint_2d(path, step, E, nu, eps_field, sig_field, eps_mac, sig_mac, pixel, fmt=None):
    """mgkmc/linear_elastic_simulator.py:568-586 save_checkpoint_2d."""
    nx, ny = np.shape(E)
    return write(path, {"fields/eps_field": eps_field, "fields/sig_field": sig_field, "fields/E_field": E,
                        "fields/nu_field": nu, "macro/eps_macro": eps_mac, "macro/sig_macro": sig_mac},
                 {"metadata": {"nx": nx, "ny": ny, "pixel": pixel, "step": step}}, fmt)


def save_checkpoint_3d(path, step, E, nu, eps_field, sig_field, eps_mac, sig_mac, pixel, fmt=None):
    """mgkmc/linear_elastic_simulator.py:588-604 save_checkpoint_3d."""
    nx, ny, nz = np.shape(E)
    return write(path, {"fields/eps_field": eps_field, "fields/sig_field": sig_field, "fields/E_field": E,
                        "fields/nu_field": nu, "macro/eps_macro": eps_mac, "macro/sig_macro": sig_mac},
                 {"metadata": {"nx": nx, "ny": ny, "nz": nz, "pixel": pixel, "step": step}}, fmt)


def _rng_state_json(rng):
    return json.dumps(rng.bit_generator.state)


def _rng_from_json(s):
    st = json.loads(s)
    bg = getattr(np.random, st["bit_generator"])()
    bg.state = st
    return np.random.Generator(bg)


def save_trajectory(path, sim, rng, step=None, fmt=None, pixel=1.0):
    """Checkpoint of a device-resident KMC/AQS trajectory (``Kmc2D``, or
    ``Kmc3D``: the reference's own 3D layout) between AQS steps, in the
    layout of mgkmc/aqs.py:1207-1267 plus the ``resume`` group.  ``rng`` is
    the Generator the trajectory draws from."""
    st = sim.state_dict()
    p = sim.p
    three_d = hasattr(sim, "nz")
    shape = (sim.nx, sim.ny, sim.nz) if three_d else (sim.nx, sim.ny)
    M = sim.M
    groups = {"fields/eps_field": st["eps"], "fields/sig_field": st["sig"], "fields/E_field": st["E"],
              "fields/nu_field": st["nu"], "fields/Tlocal": np.full(shape, float(p["T"])),
              "grid/eps_plastic": st["eps_p"], "grid/soft_prop": st["soft"], "grid/Q": st["Q"],
              "grid/Q0": st["Q0"], "grid/catalog": st["catalog"], "grid/last_event_time": st["t_last"],
              "state/eps_macro": st["eps_macro"], "resume/prev_strain_dir": st["prev"]}
    nsite = 4 if three_d else 3  # (x, y, [z,] m) per flip
    ev = np.array([e[:nsite] for e in st["events"]], dtype=np.int32).reshape(-1, nsite)
    groups["history/flips"] = ev
    groups["resume/event_times"] = np.array([e[nsite] for e in st["events"]], dtype=np.float64)
    meta = {"nx": sim.nx, "ny": sim.ny, "nz": sim.nz if three_d else 1, "M": M, "gamma0": p["gamma0"],
            "pixel": pixel, "timestamp": datetime.datetime.now().isoformat(),
            "step": int(st["steps_done"] if step is None else step), "sim_time": st["time"], "nu0": p["nu0"],
            "temperature": p["T"], "strain_rate": p["strain_rate"], "jp": p["jp"], "jt": p["jt"],
            "neighbor_softening_fraction": p["jn"], "softening_cap": p["cap"], "softening_scheme": 0,
            "scale_rate_by_volume": True, "enable_thermal": False}
    if hasattr(sim, "stability_threshold"):
        meta["stability_threshold"] = sim.stability_threshold
    resume = {"steps_done": int(st["steps_done"]), "n_solves": int(st["n_solves"]),
              "rng_state": _rng_state_json(rng), "selection": sim.selection, "ls_start": sim.ls_start,
              "precision": getattr(sim.ls, "precision", "fp64"), "unit_ready": int(st.get("unit_ready", 0)),
              "flips_since_sync": int(st.get("flips_since_sync", 0))}
    return write(path, groups, {"metadata": meta, "resume": resume}, fmt)


def load_trajectory(path):
    """(state dict for ``Kmc2D.load_state_dict`` or ``Kmc3D.load_state_dict``,
    numpy Generator, metadata)."""
    data, attrs = load(path)
    meta, res = attrs.get("metadata", {}), attrs.get("resume", {})
    ev = data["history/flips"]
    nsite = ev.shape[1] if ev.ndim == 2 else 3
    times = data["resume/event_times"]
    st = {"eps": data["fields/eps_field"], "sig": data["fields/sig_field"], "E": data["fields/E_field"],
          "nu": data["fields/nu_field"], "eps_p": data["grid/eps_plastic"], "soft": data["grid/soft_prop"],
          "Q": data["grid/Q"], "Q0": data["grid/Q0"], "catalog": data["grid/catalog"],
          "t_last": data["grid/last_event_time"], "prev": data["resume/prev_strain_dir"],
          "eps_macro": data["state/eps_macro"], "time": float(meta["sim_time"]),
          "steps_done": int(res["steps_done"]), "n_solves": int(res["n_solves"]),
          "unit_ready": bool(res.get("unit_ready", 0)), "flips_since_sync": int(res.get("flips_since_sync", 0)),
          "events": [tuple(int(v) for v in e) + (float(t),) for e, t in zip(ev.reshape(-1, nsite), times)]}
    rng = _rng_from_json(str(res["rng_state"]))
    return st, rng, meta
