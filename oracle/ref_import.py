"""Import shim for the unmodified mgkmc reference package (test infrastructure).

The reference imports ``pyfftw``, ``h5py``, ``meshio`` and ``matplotlib`` at
module level (mgkmc/fft.py:3-7, mgkmc/analysis/vtk.py:2,
mgkmc/analysis/history.py:10, mgkmc/analysis/plotting.py).  None of them is
needed by the hot path, and only ``pyfftw`` carries arithmetic: its
``interfaces.numpy_fft`` functions are drop-in replacements of ``numpy.fft``
with an extra ``threads=`` keyword.  This shim maps them onto ``numpy.fft``
(pocketfft) with ``threads`` dropped, and gives the I/O modules empty stubs.

FFTW itself (unpinned in the reference's requirements.txt:5) is therefore
replaced by pocketfft; both are exact-to-roundoff DFTs and no reference test
pins FFT output bits.
"""
import os
import sys
import types

import numpy as np


def _wrap(fn):
    def inner(*args, threads=None, **kw):
        kw.pop("planner_effort", None)
        kw.pop("overwrite_input", None)
        return fn(*args, **kw)
    return inner


def install_stubs():
    """Install the pyfftw/h5py/meshio/matplotlib stand-ins into sys.modules."""
    if "pyfftw" in sys.modules and getattr(sys.modules["pyfftw"], "_mgkmc_stub", False):
        return
    pyfftw = types.ModuleType("pyfftw")
    pyfftw._mgkmc_stub = True
    pyfftw.config = types.SimpleNamespace(NUM_THREADS=1, PLANNER_EFFORT="FFTW_ESTIMATE")
    interfaces = types.ModuleType("pyfftw.interfaces")
    cache = types.ModuleType("pyfftw.interfaces.cache")
    cache.enable = lambda *a, **k: None
    cache.set_keepalive_time = lambda *a, **k: None
    npfft = types.ModuleType("pyfftw.interfaces.numpy_fft")
    for name in ("fft", "ifft", "fft2", "ifft2", "fftn", "ifftn", "rfft", "irfft",
                 "rfftn", "irfftn", "rfft2", "irfft2"):
        setattr(npfft, name, _wrap(getattr(np.fft, name)))
    npfft.fftfreq = np.fft.fftfreq
    npfft.rfftfreq = np.fft.rfftfreq
    npfft.fftshift = np.fft.fftshift
    npfft.ifftshift = np.fft.ifftshift
    interfaces.cache = cache
    interfaces.numpy_fft = npfft
    pyfftw.interfaces = interfaces
    builders = types.ModuleType("pyfftw.builders")
    pyfftw.builders = builders
    sys.modules["pyfftw"] = pyfftw
    sys.modules["pyfftw.interfaces"] = interfaces
    sys.modules["pyfftw.interfaces.cache"] = cache
    sys.modules["pyfftw.interfaces.numpy_fft"] = npfft
    sys.modules["pyfftw.builders"] = builders
    for name in ("h5py", "meshio"):
        if name not in sys.modules:
            sys.modules[name] = types.ModuleType(name)
    if "matplotlib" not in sys.modules:
        mpl = types.ModuleType("matplotlib")
        mpl.use = lambda *a, **k: None
        plt = types.ModuleType("matplotlib.pyplot")
        mpl.pyplot = plt
        sys.modules["matplotlib"] = mpl
        sys.modules["matplotlib.pyplot"] = plt


def import_reference(path=None):
    """Import the reference ``mgkmc`` package from ``path`` (default: the
    environment variable ``MGKMC_REFERENCE``; one of the two is required)."""
    install_stubs()
    path = path or os.environ.get("MGKMC_REFERENCE")
    if not path:
        raise FileNotFoundError("reference checkout not given: pass a path or set MGKMC_REFERENCE")
    if not os.path.isdir(os.path.join(path, "mgkmc")):
        raise FileNotFoundError(f"reference package not found under {path}")
    if path not in sys.path:
        sys.path.insert(0, path)
    import mgkmc  # noqa: F401
    return mgkmc
