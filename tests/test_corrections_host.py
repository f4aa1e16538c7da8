"""Host-built correction transfers against the oracle's float64 restatements
(corrections/window.py:229-265, corrections/pgd.py:154-237,
corrections/softening.py:49-80) and the combined correction's kernel selection
(corrections/core.py:396-422).  Tables are built on the CPU here; the force
runs them on the GPU in tests/test_gpu_force.py."""
import numpy as np
import pytest

from oracle import pm as opm


def _confs(ptcl=(16, 16, 16), mesh=2):
    import pmpp_b200 as pb
    return pb, pb.Configuration(4.0, ptcl, mesh, device="cpu"), opm.Conf(4.0, ptcl, mesh_shape=mesh)


@pytest.mark.parametrize("kw,a", [({}, 1.0), (dict(alpha0=-0.4, A=0.3, B=-0.2, kl=0.2, ks=0.8), 0.35),
                                  (dict(pgd_alpha0=0.25, pgd_kl=0.05, pgd_ks=1.5), 0.7)])
def test_pgd_transfer_matches_oracle(kw, a):
    pb, conf, co = _confs()
    from pmpp_b200.corrections import init_potential_correction
    c = init_potential_correction("pgd", **kw)
    T, R = c.transfer_tables(a, None, conf)
    assert R is None and T.shape == (32, 32, 17)
    args = dict(alpha0=kw.get("alpha0", kw.get("pgd_alpha0", 0.1)), A=kw.get("A", 0.0), B=kw.get("B", 0.0),
                kl=kw.get("kl", kw.get("pgd_kl", 0.1)), ks=kw.get("ks", kw.get("pgd_ks", 1.0)))
    ref = opm.pgd_transfer(co, a, **args)
    np.testing.assert_allclose(T.numpy(), ref, rtol=0, atol=2e-6)
    assert T.numpy()[0, 0, 0] == 1.0  # no band at k = 0
    # alpha(a) per scale factor: a second a gives a second table
    T2, _ = c.transfer_tables(0.5 * a, None, conf)
    np.testing.assert_allclose(T2.numpy(), opm.pgd_transfer(co, 0.5 * a, **args), rtol=0, atol=2e-6)


@pytest.mark.parametrize("mode", ["smoothstep", "linear"])
@pytest.mark.parametrize("strength,start,stop", [(0.6, 0.7, 1.0), (2.5, 0.2, 0.9), (0.3, 0.45, 0.55)])
def test_softening_transfer_matches_oracle(mode, strength, start, stop):
    pb, conf, co = _confs(mesh=3)
    from pmpp_b200.corrections import init_potential_correction
    c = init_potential_correction("softening", softening_strength=strength, softening_start=start,
                                  softening_stop=stop, softening_mode=mode)
    T, _ = c.transfer_tables(1.0, None, conf)
    ref = opm.softening_transfer(co, strength, start, stop, mode)
    np.testing.assert_allclose(T.numpy(), ref, rtol=0, atol=2e-6)
    assert T.min() >= 0.0


def test_unknown_softening_mode_and_model_raise():
    from pmpp_b200.corrections import init_potential_correction
    with pytest.raises(ValueError, match="high-k softening mode"):
        init_potential_correction("softening", mode="cubic")
    with pytest.raises(ValueError, match="Unsupported correction model"):
        init_potential_correction("mesh_cnn_typo")


@pytest.mark.parametrize("model", ["windowed_pgd", "pm_window+pgd", "pgd_window"])
def test_windowed_pgd_is_the_product(model):
    pb, conf, co = _confs()
    from pmpp_b200.corrections import init_potential_correction
    c = init_potential_correction(model, window_alpha=0.3, window_max_gain=3.0, pgd_alpha0=0.2, pgd_ks=0.9)
    assert c.green_kernel == 1 and c.gradient_kernel == "spectral"
    T, _ = c.transfer_tables(0.6, None, conf)
    ref = opm.window_gain(co, alpha=0.3, max_gain=3.0) * opm.pgd_transfer(co, 0.6, alpha0=0.2, ks=0.9)
    np.testing.assert_allclose(T.numpy(), ref, rtol=2e-6, atol=2e-6)


def test_windowed_softening_and_gradient_selection():
    pb, conf, co = _confs()
    from pmpp_b200.corrections import (CombinedPotentialCorrection, HighKSofteningCorrection, PMWindowCompensation,
                                       init_potential_correction)
    c = init_potential_correction("pm_window+softening", strength=0.5, window_gradient_kernel="fastpm_4point",
                                  green_kernel="continuum")
    assert c.green_kernel == 0 and c.gradient_kernel == "fastpm_4point"
    T, _ = c.transfer_tables(1.0, None, conf)
    ref = opm.window_gain(co) * opm.softening_transfer(co, 0.5)
    np.testing.assert_allclose(T.numpy(), ref, rtol=2e-6, atol=2e-6)
    # the non-continuum Green's function and the one non-spectral derivative win
    w = PMWindowCompensation(alpha=0.0, green_kernel="discrete_laplacian")
    s = HighKSofteningCorrection(strength=0.1)
    assert CombinedPotentialCorrection(window=w, softening=s).green_kernel == 1
    assert CombinedPotentialCorrection(window=w, softening=s).transfer_tables(1.0, None, conf)[0] is not None

    class Other:
        green_kernel = 0
        gradient_kernel = "finite_difference"

        def transfer_tables(self, a, cosmo, conf):
            return None, None

    w4 = PMWindowCompensation(gradient_kernel="fastpm_4point")
    with pytest.raises(ValueError, match="incompatible force-gradient kernels"):
        CombinedPotentialCorrection(window=w4, pgd=Other())
