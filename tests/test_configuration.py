"""Configuration contracts (no GPU), restated from the reference's
tests/test_deep_configuration_contracts.py:11-37, 47-93, 114-123 for the
single-device options this package implements (no observers, Pallas or
multi-GPU fields)."""
import math

import numpy as np
import pytest

import pmpp_b200 as pb


@pytest.mark.parametrize("kwargs, message", [
    ({"ptcl_grid_shape": (4, 4, 4), "mesh_shape": (4, 4)}, "dimensions differ"),
    ({"ptcl_grid_shape": (4, 4, 4), "mesh_shape": (2, 2, 2)}, "cannot be smaller"),
    ({"ptcl_grid_shape": (4, 2, 2), "mesh_shape": (8, 5, 4)}, "aspect ratios differ"),
    ({"symp_splits": ((0.5, 0.5, 0.0), (0.5, 0.5))}, "not supported"),
    ({"symp_splits": ((0.2, 0.5), (0.2, 0.5))}, "symplectic splits"),
])
def test_rejects_inconsistent_shapes_and_integrators(kwargs, message):
    args = {"ptcl_spacing": 1.0, "ptcl_grid_shape": (4, 4, 4), "mesh_shape": 1, "device": "cpu"}
    args.update(kwargs)
    with pytest.raises(ValueError, match=message):
        pb.Configuration(**args)


def test_schedules_and_derived_units():
    conf = pb.Configuration(2.5, (2, 3, 4), mesh_shape=(4, 6, 8), a_start=0.2, a_stop=0.8, a_lpt_maxstep=0.07,
                            a_nbody_maxstep=0.21, a_custom=[0.2, 0.31, 0.8],
                            growth_a_custom=np.asarray([0.0, 0.2, 0.8]), device="cpu")
    assert conf.a_custom == (0.2, 0.31, 0.8)
    assert conf.growth_a_custom == (0.0, 0.2, 0.8)
    np.testing.assert_allclose(conf.a_nbody, [0.2, 0.31, 0.8])
    np.testing.assert_allclose(conf.growth_a, [0.0, 0.2, 0.8])
    assert conf.a_lpt_num == 3 and conf.a_nbody_num == 3
    assert conf.a_lpt_step <= 0.07 and conf.a_nbody_step <= 0.21 + 1e-12
    assert conf.ptcl_num == 24 and conf.ptcl_cell_vol == 2.5**3
    assert conf.box_size == (5.0, 7.5, 10.0) and conf.box_vol == 375.0
    assert conf.cell_size == 1.25 and conf.disp_size == 0.8 and conf.mesh_size == 192
    assert conf.local_mesh_size == 192
    assert conf.V == conf.L / conf.T
    assert conf.H_0 == conf.H_0_SI * conf.T
    assert conf.c == conf.c_SI / conf.V
    assert conf.G == conf.G_SI * conf.M / (conf.L * conf.V**2)
    np.testing.assert_allclose(conf.rho_crit, 3 * conf.H_0**2 / (8 * np.pi * conf.G), rtol=1e-12)
    # code units: H_0 = 1 in [1/T], c in units of 100 km/s
    assert math.isclose(conf.H_0, 1.0, rel_tol=1e-15) and math.isclose(conf.c, 2997.92458, rel_tol=1e-12)
    assert conf.transfer_k_num > 2 and conf.transfer_lgk_step <= conf.transfer_lgk_maxstep
    assert conf.transfer_k[0] == 0 and conf.transfer_k.shape == (conf.transfer_k_num, )


def test_single_device_attributes():
    conf = pb.Configuration(1.0, (2, 2, 2), mesh_shape=2, device="cpu")
    assert conf.use_mGPU is False
    assert conf.local_mesh_shape == conf.mesh_shape == conf.local_mesh_with_halo_shape
    assert conf.mesh_halo_width == 0 and conf.ptcl_halo_width == 0
    with pytest.raises(AttributeError, match="definitely_missing"):
        _ = conf.definitely_missing


def test_generated_schedules_without_custom_grids():
    conf = pb.Configuration(1.0, (2, 2, 2), mesh_shape=1, a_start=0.1, a_stop=0.4, a_lpt_maxstep=0.04,
                            a_nbody_maxstep=0.11, device="cpu")
    assert conf.a_custom is None and conf.growth_a_custom is None
    np.testing.assert_allclose(np.diff(conf.a_lpt), conf.a_lpt_step, rtol=1e-6, atol=1e-7)
    np.testing.assert_allclose(np.diff(conf.a_nbody), conf.a_nbody_step, rtol=1e-6, atol=1e-7)
    np.testing.assert_allclose(conf.growth_a, np.concatenate((conf.a_lpt, conf.a_nbody[1:])))


def test_custom_growth_grid_feeds_the_growth_table():
    a_nb = np.linspace(0.1, 1.0, 6)
    conf = pb.Configuration(4.0, (8, 8, 8), 1, a_start=0.1, a_custom=a_nb, device="cpu")
    ref = pb.boltzmann(pb.SimpleLCDM(conf))
    custom = pb.Configuration(4.0, (8, 8, 8), 1, a_start=0.1, a_custom=a_nb, growth_a_custom=conf.growth_a,
                              device="cpu")
    c = pb.boltzmann(pb.SimpleLCDM(custom))
    np.testing.assert_array_equal(custom.growth_a, conf.growth_a)
    np.testing.assert_array_equal(c.growth, ref.growth)
