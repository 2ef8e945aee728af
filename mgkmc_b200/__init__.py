"""B200-native mechanical-equilibrium hot path of mgkmc.

Hand-written sm_100a CUDA kernels behind a C-ABI (include/mgkmc.h, built into
``libmgkmc_cuda.so``), with Python host code that keeps the reference's
function names and arguments:

* ``linear_elastic_simulator.spectral_solver_2d`` -- mgkmc/linear_elastic_simulator.py:12
* ``kmc_simulator_functions.compute_barrier_2d / compute_rates_2d /
  select_event_2d / decode_index_2d / apply_flip_soa_2d`` -- mgkmc/kmc_simulator_functions.py
"""
from . import _lib  # noqa: F401

__all__ = ["build", "linear_elastic_simulator", "kmc_simulator_functions", "workloads"]
