"""Host FP64 cosmology (native library) against the oracle restatement."""
import numpy as np

from oracle import cosmology as ocos
from oracle import pm as opm


def _pair(a_custom=np.linspace(0.1, 1, 11)):
    import pmpp_b200 as pb
    co = opm.Conf(4.0, (16, 16, 16), mesh_shape=2, a_start=0.1, a_custom=a_custom)
    conf = pb.Configuration(4.0, (16, 16, 16), 2, a_start=0.1, a_custom=a_custom, device="cpu")
    return pb, co, conf


def test_growth_table_matches_oracle():
    pb, co, conf = _pair()
    c = pb.boltzmann(pb.SimpleLCDM(conf))
    oc = opm.boltzmann(ocos.Cosmo(), co)
    assert np.abs(c.growth - oc.growth).max() < 1e-9
    assert np.abs(c.transfer - oc.transfer).max() < 1e-14


def test_growth_matter_era_normalisation():
    """D(a) -> a deep in matter domination (boltzmann.py growth IC (1, 0, 3/7, 0))."""
    pb, co, conf = _pair()
    c = pb.boltzmann(pb.SimpleLCDM(conf))
    a = 1e-3
    np.testing.assert_allclose(float(pb.growth(a, c)) / a, 1.0, rtol=1e-3)
    np.testing.assert_allclose(float(pb.growth(a, c, order=2)) / a**2, 3 / 7, rtol=2e-3)


def test_time_factors_and_omega_m_derivative():
    pb, co, conf = _pair()
    c = pb.boltzmann(pb.SimpleLCDM(conf))
    oc = opm.boltzmann(ocos.Cosmo(), co)
    for args in [(0.19, 0.19, 0.235), (0.28, 0.19, 0.37), (0.1, 0.1, 0.145)]:
        f, df = c.kick_factor(*args, with_grad=True)
        np.testing.assert_allclose(f, opm.kick_factor(*args, oc, co), rtol=1e-8)
        np.testing.assert_allclose(df, opm._factor_dOm(opm.kick_factor, args, oc, co), rtol=1e-4)
        f, df = c.drift_factor(*args, with_grad=True)
        np.testing.assert_allclose(f, opm.drift_factor(*args, oc, co), rtol=1e-8)
        np.testing.assert_allclose(df, opm._factor_dOm(opm.drift_factor, args, oc, co), rtol=1e-4)


def test_sigma8_normalisation():
    pb, co, conf = _pair()
    c = pb.Cosmology.from_sigma8(conf, 0.8, n_s=0.96, Omega_m=0.3, Omega_b=0.05, h=0.7)
    np.testing.assert_allclose(c.sigma8, 0.8, rtol=1e-10)
    oc = opm.cosmo_from_sigma8(co, 0.8, n_s=0.96, Omega_m=0.3, Omega_b=0.05, h=0.7)
    np.testing.assert_allclose(c.A_s_1e9, oc.A_s_1e9, rtol=1e-8)


def test_linear_power_matches_oracle():
    pb, co, conf = _pair()
    c = pb.boltzmann(pb.SimpleLCDM(conf))
    oc = opm.boltzmann(ocos.Cosmo(), co)
    k = np.geomspace(1e-3, 5, 50)
    np.testing.assert_allclose(pb.linear_power(k, None, c), ocos.linear_power(k, None, oc, co.transfer_k), rtol=1e-12)


def test_transfer_and_varlin_helpers():
    """transfer / varlin (boltzmann.py:140-174, 314-355): table interpolation,
    sigma8 consistency and growth scaling; both refuse an empty table."""
    import pytest
    from pmpp_b200 import cosmology as C
    pb, co, conf = _pair()
    c = pb.boltzmann(pb.SimpleLCDM(conf))
    tk = conf.transfer_k
    np.testing.assert_array_equal(C.transfer(tk[10:20], c), c.transfer[10:20])
    mid = np.sqrt(tk[10] * tk[11])
    assert min(c.transfer[10], c.transfer[11]) <= C.transfer(mid, c) <= max(c.transfer[10], c.transfer[11])
    np.testing.assert_allclose(np.sqrt(C.varlin(8.0, 1.0, c)), c.sigma8, rtol=1e-12)
    s2 = C.varlin(np.array([4.0, 8.0, 16.0]), None, c)
    assert s2.shape == (3, ) and np.all(np.diff(s2) < 0)
    np.testing.assert_allclose(C.varlin(8.0, 0.5, c), s2[1] * float(pb.growth(0.5, c))**2, rtol=1e-12)
    bare = pb.SimpleLCDM(conf)
    with pytest.raises(ValueError):
        C.transfer(tk[:3], bare)
    with pytest.raises(ValueError):
        C.varlin(8.0, 1.0, bare)


def test_cosmology_param_helpers():
    """models.py:267-329: names include set optional parameters, values follow
    the names, replace returns a new instance."""
    from pmpp_b200 import cosmology as C
    pb, co, conf = _pair()
    c = pb.SimpleLCDM(conf)
    assert C.cosmology_param_names(c) == ("A_s_1e9", "n_s", "Omega_m", "Omega_b", "h")
    w = c.replace(w_0_=-0.9, Omega_k_=0.01)
    assert C.cosmology_param_names(w) == ("A_s_1e9", "n_s", "Omega_m", "Omega_b", "h", "Omega_k_", "w_0_")
    assert C.cosmology_param_values(w) == (2.0, 0.96, 0.3, 0.05, 0.7, 0.01, -0.9)
    assert C.cosmology_param_values(w, ("h", "Omega_m")) == (0.7, 0.3)
    r = C.replace_cosmology_params(c, ("Omega_m", "h"), (0.31, 0.68))
    assert (r.Omega_m, r.h, c.Omega_m, c.h) == (0.31, 0.68, 0.3, 0.7)


def test_boltzmann_contracts():
    """Restated from the reference's tests/test_deep_boltzmann_contracts.py:19-53:
    both Eisenstein-Hu fits are exactly 1 at k = 0, the no-wiggle fit is finite,
    non-increasing and within 2e-3 of the baryonic one on large scales (and
    matches the oracle); missing tables fail explicitly; switched-off
    components stay unset; variance scales with D(a)^2."""
    import pytest
    from pmpp_b200 import cosmology as C
    import pmpp_b200 as pb
    conf = pb.Configuration(10.0, (8, 8, 8), 1, a_start=1 / 64, a_nbody_maxstep=1 / 64, device="cpu")
    smooth_conf = pb.Configuration(10.0, (8, 8, 8), 1, a_start=1 / 64, a_nbody_maxstep=1 / 64,
                                   transfer_fit_nowiggle=True, device="cpu")
    cosmo = pb.SimpleLCDM(conf)
    k = np.concatenate(([0.0], np.geomspace(1e-4, 0.5, 64)))
    baryonic = C.transfer_fit(k, cosmo, conf)
    smooth = C.transfer_fit(k, cosmo, smooth_conf)
    assert np.all(np.isfinite(smooth)) and smooth[0] == 1 and baryonic[0] == 1
    np.testing.assert_allclose(smooth[1], baryonic[1], rtol=2e-3, atol=2e-6)
    assert np.all(np.diff(smooth) <= 1e-12)
    np.testing.assert_allclose(smooth, ocos.transfer_fit(k, ocos.Cosmo(), nowiggle=True), rtol=1e-13, atol=1e-15)
    empty = pb.SimpleLCDM(conf)
    with pytest.raises(ValueError, match="Transfer table is empty"):
        C.transfer(np.asarray([0.1]), empty, conf)
    with pytest.raises(ValueError, match="Growth table is empty"):
        C.growth(0.5, empty, conf)
    with pytest.raises(ValueError, match="variance table is empty"):
        C.varlin(1.0, None, empty, conf)
    disabled = C.boltzmann(empty, conf, transfer=False, growth=False, varlin=False)
    assert disabled.transfer is None and disabled.growth is None
    complete = C.boltzmann(empty, conf)
    radius = np.asarray([5.0, 10.0, 20.0])
    np.testing.assert_allclose(C.varlin(radius, 0.4, complete, conf),
                               C.varlin(radius, None, complete, conf) * C.growth(0.4, complete, conf)**2,
                               rtol=2e-14, atol=0)
    with pytest.raises(ValueError, match="dim=2 not supported"):
        import types
        C.linear_power(np.asarray([0.1]), None, complete, types.SimpleNamespace(dim=2))
