"""CPU-side checks of the C-ABI library: it loads and exports every symbol
the public header declares (no compute call without a GPU)."""
import ctypes

from mgkmc_b200 import _lib as L


def test_library_exports_every_declared_symbol():
    lib = L.lib()
    declared = L.declared_symbols()
    assert len(declared) >= 10
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing
    # every declared symbol has a ctypes signature in the binding
    assert set(declared) <= set(L._SIGS), set(declared) - set(L._SIGS)


def test_host_only_entry_points():
    lib = L.lib()
    assert lib.mgk_version() >= 100
    assert lib.mgk_status_string(0) == b"ok"
    for n in (1, 2, 3, 4, 6, 8, 9, 12, 64, 96, 192, 256, 384, 768, 1024, 4096):
        assert lib.mgk_fft_supported(n) == 1, n
    for n in (0, 5, 7, 10, 8192):
        assert lib.mgk_fft_supported(n) == 0, n
    assert lib.mgk_kmc_rates_work_bytes(524288) >= 4 * 2048


def test_bad_arguments_are_rejected_without_a_device():
    lib = L.lib()
    h = ctypes.c_void_p()
    assert lib.mgk_ls2d_create(30, 64, 0, 0, ctypes.byref(h)) == L.BAD_ARG  # 30 = 2*3*5
    assert lib.mgk_ls2d_create(9, 64, 0, 0, ctypes.byref(h)) == L.BAD_ARG   # rows are paired: nx even
    assert b"unsupported" in lib.mgk_last_error()
    assert lib.mgk_ls2d_create(64, 64, 7, 0, ctypes.byref(h)) == L.BAD_ARG
    assert lib.mgk_kmc_select(None, None, None, 0.5, None, None) == L.BAD_ARG


def test_new_entry_points_reject_bad_arguments_without_a_device():
    # argument checks of the patch, Anderson and law entry points run before
    # any device work
    lib = L.lib()
    assert lib.mgk_aa_work_bytes(1 << 20) == 296 * 16 * 8
    assert lib.mgk_aa_update(0, None, None, None, 5, 0, 0, 0, None, None, None) == L.BAD_ARG
    one = ctypes.c_void_p(16)  # never dereferenced: the size checks fail first
    assert lib.mgk_aa_update(10, one, one, one, 9, 0, 0, 0, one, one, None) == L.BAD_ARG  # m > 8
    assert lib.mgk_aa_mix(10, one, one, 3, 4, one, one, None) == L.BAD_ARG  # ncols > m
    assert lib.mgk_kmc2d_patch(0, 4, 2, None, None, 0.0, None, None, 3, None, None, None, None) == L.BAD_ARG
    assert lib.mgk_kmc2d_patch_setup(8, 8, 5000, one, one, one, one, None) == L.BAD_ARG  # R > 4096
    assert lib.mgk_ls3d_set_secant(None, 0.5, 10.0) == L.BAD_ARG
    assert lib.mgk_ls2d_set_landau(None, None, 0, 0.0, 0.1, 1.0, 0) == L.BAD_ARG
    assert lib.mgk_ls2d_set_e33_out(None, 0, None) == L.BAD_ARG


def test_landau_refusals_before_device_work():
    import numpy as np
    import pytest
    from mgkmc_b200 import linear_elastic_simulator as les
    lam = np.full((8, 8), 4e10)
    mu = np.full((8, 8), 3e10)
    v = dict(v1=0.0, v2=0.0, v3=0.0, g1=0.0, g2=0.0, g3=0.0, g4=0.0)
    eb = np.zeros((2, 2))
    with pytest.raises(ValueError):
        les.spectral_solver_landau_2d(lam, mu, **v, eps_bar=eb, plane_mode="plane_strian")
    with pytest.raises(NotImplementedError):
        les.spectral_solver_landau_2d(lam, mu, **v, eps_bar=eb, solver="newton_cg")
    with pytest.raises(NotImplementedError):
        les.spectral_solver_landau_2d(lam, mu, **v, eps_bar=eb, anderson_m=9)
