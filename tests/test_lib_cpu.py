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
