"""CPU oracle for the mgkmc mechanical-equilibrium hot path.

TEST INFRASTRUCTURE ONLY.  Nothing in this package is part of the product:
only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` may import it, and there only as the
checker (or as the timed CPU restatement of the reference), never as a code
path that produces results for a user.  The CUDA library ``mgkmc_b200`` has no
CPU fallback and fails loudly when its extension is missing.

Modules
-------
``ls``      numpy restatement of the small-strain Lippmann-Schwinger solver
            (mgkmc/linear_elastic_simulator.py:12-88, :274-376) and of its
            mixed-BC macro loop (:176-197).
``kmc``     numpy restatement of the per-voxel STZ kernels
            (mgkmc/kmc_simulator_functions.py:5-218, mgkmc/stz/*.py).
``fs``      numpy restatement of the de Geus finite-strain Newton-Krylov
            step in 3D (mgkmc/finite_strain_simulator.py:2967-3168) with
            SVK and a 3D Neo-Hookean law.
``ref_import``  an import shim that makes the unmodified reference package
            importable in a container without pyfftw/h5py/meshio/matplotlib
            (pyfftw's numpy interface is mapped to ``numpy.fft``).  Used only by
            the golden-fixture generator, never on the GPU host.

Parity is pinned: ``tests/golden/make_golden.py`` runs the unmodified
reference functions on seeded inputs and stores their outputs as fixtures;
``tests/test_oracle_golden.py`` checks every restatement here against them.
"""
