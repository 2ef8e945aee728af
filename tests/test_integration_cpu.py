"""patch_reference: the reference's hot-path names (driver-module bindings
and the names its drivers import at call time) are redirected to the drop-ins
and restored, checked on a stand-in package with the reference's module
layout (no device needed); with MGKMC_REFERENCE set, on the real package."""
import os
import types

import pytest

from mgkmc_b200 import integration as I


def _fake_package():
    pkg = types.SimpleNamespace()
    for mod_name, attr, _ in I._TABLE:
        parts = mod_name.split(".")
        obj = pkg
        for p in parts:
            if not hasattr(obj, p):
                setattr(obj, p, types.SimpleNamespace())
            obj = getattr(obj, p)
        setattr(obj, attr, ("original", mod_name, attr))
    return pkg


def test_patch_and_restore_on_stand_in():
    pkg = _fake_package()
    done = I.patch_reference(pkg)
    assert len(done) == len(I._TABLE)
    assert pkg.kmc_simulator.apply_flip_soa_2d is I._kf.apply_flip_soa_2d
    assert pkg.linear_elastic_simulator.linear_elastic_simulation_2d is I._les.linear_elastic_simulation_2d
    assert pkg.finite_strain_simulator.finite_strain_solver_step_2d is I._fss.finite_strain_solver_step_2d
    assert pkg.stz.update_fft.update_stress_fft_full is I._les.update_stress_fft_full
    I.unpatch_reference()
    assert pkg.kmc_simulator.apply_flip_soa_2d == ("original", "kmc_simulator", "apply_flip_soa_2d")
    assert pkg.aqs.compute_rates == ("original", "aqs", "compute_rates")


@pytest.mark.skipif(not os.environ.get("MGKMC_REFERENCE"), reason="reference checkout not given")
def test_patch_real_reference():
    from oracle.ref_import import import_reference
    mgkmc = import_reference()
    done = I.patch_reference(mgkmc)
    try:
        import mgkmc.kmc_simulator as ks
        import mgkmc.linear_elastic_simulator as les
        assert ks.select_event_2d is I._kf.select_event_2d
        assert les.linear_elastic_simulation_3d is I._les.linear_elastic_simulation_3d
        assert les.landau_elastic_simulation_3d is I._les.landau_elastic_simulation_3d
        assert "aqs.apply_flip_soa" in done
    finally:
        I.unpatch_reference()
