"""Redirects the reference package's hot-path names to the B200 drop-ins.

The reference's drivers resolve their solvers and KMC kernels through module
attributes: names bound at import time in the driver modules
(mgkmc/kmc_simulator.py:6-10, mgkmc/aqs.py:6-13) and names imported at call
time from their defining modules (run.py:483, :729, :783, :934;
kmc_simulator.py:403-418, :479).  ``patch_reference(mgkmc)`` replaces both
kinds, so KmcSimulation2D, ThermalSimulation and run.py run their hot path on
the GPU without edits; ``unpatch_reference`` restores the originals.

    import mgkmc
    from mgkmc_b200.integration import patch_reference
    patch_reference(mgkmc)
"""
import importlib

from . import finite_strain_simulator as _fss
from . import kmc_simulator_functions as _kf
from . import linear_elastic_simulator as _les
from . import stz as _stz
from . import vtk as _vtk

# (reference module, attribute) -> replacement
_TABLE = [
    # drivers' import-time bindings
    ("kmc_simulator", "spectral_solver_2d", _les.spectral_solver_2d),                # :517
    ("kmc_simulator", "spectral_solver_secant_2d", _les.spectral_solver_secant_2d),  # :454
    ("kmc_simulator", "spectral_solver_rose_2d", _les.spectral_solver_rose_2d),      # :465
    ("kmc_simulator", "compute_barrier_2d", _kf.compute_barrier_2d),                 # :529
    ("kmc_simulator", "compute_rates_2d", _kf.compute_rates_2d),                     # :891
    ("kmc_simulator", "select_event_2d", _kf.select_event_2d),                       # :899
    ("kmc_simulator", "decode_index_2d", _kf.decode_index_2d),                       # :900
    ("kmc_simulator", "apply_flip_soa_2d", _kf.apply_flip_soa_2d),                   # :1025
    ("aqs", "update_stress_fft_full", _les.update_stress_fft_full),                  # :349
    ("aqs", "compute_barrier", _stz.compute_barrier),                                # :457
    ("aqs", "compute_rates", _stz.compute_rates),                                    # :873
    ("aqs", "select_event", _stz.select_event),                                      # :889
    ("aqs", "decode_index", _stz.decode_index),                                      # :892
    ("aqs", "apply_flip_soa", _stz.apply_flip_soa),                                  # :996
    # names the drivers import at call time from their defining modules
    ("linear_elastic_simulator", "spectral_solver_2d", _les.spectral_solver_2d),
    ("linear_elastic_simulator", "spectral_solver_3d", _les.spectral_solver_3d),
    ("linear_elastic_simulator", "spectral_solver_secant_2d", _les.spectral_solver_secant_2d),
    ("linear_elastic_simulator", "spectral_solver_secant_3d", _les.spectral_solver_secant_3d),
    ("linear_elastic_simulator", "spectral_solver_rose_2d", _les.spectral_solver_rose_2d),
    ("linear_elastic_simulator", "spectral_solver_landau_2d", _les.spectral_solver_landau_2d),
    ("linear_elastic_simulator", "spectral_solver_landau_3d", _les.spectral_solver_landau_3d),  # aqs.py:331
    ("linear_elastic_simulator", "linear_elastic_simulation_2d", _les.linear_elastic_simulation_2d),  # run.py:729
    ("linear_elastic_simulator", "linear_elastic_simulation_3d", _les.linear_elastic_simulation_3d),  # run.py:934
    ("linear_elastic_simulator", "secant_elastic_simulation_2d", _les.secant_elastic_simulation_2d),  # run.py:544
    ("linear_elastic_simulator", "rose_elastic_simulation_2d", _les.rose_elastic_simulation_2d),      # run.py:608
    ("linear_elastic_simulator", "landau_elastic_simulation_2d", _les.landau_elastic_simulation_2d),  # run.py:666
    ("linear_elastic_simulator", "secant_elastic_simulation_3d", _les.secant_elastic_simulation_3d),  # run.py:830
    ("linear_elastic_simulator", "landau_elastic_simulation_3d", _les.landau_elastic_simulation_3d),  # run.py:879
    ("finite_strain_simulator", "finite_strain_solver_step_2d", _fss.finite_strain_solver_step_2d),   # ks:403-418
    ("finite_strain_simulator", "finite_strain_solver_step_3d", _fss.finite_strain_solver_step_3d),   # aqs.py:289
    ("finite_strain_simulator", "finite_strain_simulation_3d", _fss.finite_strain_simulation_3d),     # run.py:783
    ("finite_strain_simulator", "finite_strain_simulation_2d", _fss.finite_strain_simulation_2d),     # run.py:483
    ("stz.update_fft", "update_stress_fft_full", _les.update_stress_fft_full),
    # the VTK writer the drivers bind at import time (meshio-free)
    ("kmc_simulator", "export_to_vtk", _vtk.export_to_vtk),                        # kmc_simulator.py:11
    ("linear_elastic_simulator", "export_to_vtk", _vtk.export_to_vtk),             # :9
    ("finite_strain_simulator", "export_to_vtk", _vtk.export_to_vtk),              # :28
    ("analysis.vtk", "export_to_vtk", _vtk.export_to_vtk),
]

_SAVED = {}


def _module(pkg, name):
    if hasattr(pkg, "__name__"):
        return importlib.import_module(f"{pkg.__name__}.{name}")
    obj = pkg
    for part in name.split("."):
        obj = getattr(obj, part)
    return obj


def patch_reference(pkg):
    """Replace the reference's hot-path names (see the table above); returns
    the list of "module.attribute" names replaced.  ``pkg`` is the imported
    ``mgkmc`` package (or any object with the same module attributes)."""
    done = []
    for mod_name, attr, repl in _TABLE:
        mod = _module(pkg, mod_name)
        if not hasattr(mod, attr):
            continue
        key = (id(mod), attr)
        if key not in _SAVED:
            _SAVED[key] = (mod, getattr(mod, attr))
        setattr(mod, attr, repl)
        done.append(f"{mod_name}.{attr}")
    return done


def unpatch_reference():
    """Restore every name ``patch_reference`` replaced."""
    for (_, attr), (mod, orig) in list(_SAVED.items()):
        setattr(mod, attr, orig)
    _SAVED.clear()
