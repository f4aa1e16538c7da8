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
