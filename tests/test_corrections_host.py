"""Host-built correction transfers against the oracle's float64 restatements
(corrections/window.py:229-265, corrections/pgd.py:154-237,
corrections/softening.py:49-80) and the combined correction's kernel selection
(corrections/core.py:396-422).  Tables are built on the CPU here; the force
runs them on the GPU in tests/test_gpu_force.py."""
import numpy as np
import pytest
import torch

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


def test_pgd_and_softening_reference_cases():
    """tests/test_potential_correction.py:224-275 restated: the PGD transfer is
    1 at k = 0 and 1 - alpha0 band elsewhere; softening of strength 0.2 keeps
    the transfer in [0.8, 1] and 1 below the taper."""
    import pmpp_b200 as pb
    conf = pb.Configuration(1.0, (8, 8, 8), 1, device="cpu")
    co = opm.Conf(1.0, (8, 8, 8), mesh_shape=1)
    from pmpp_b200.corrections import init_potential_correction
    p = init_potential_correction("pgd", pgd_alpha0=0.25, pgd_A=0.0, pgd_B=0.0, pgd_kl=0.5, pgd_ks=2.0)
    T, _ = p.transfer_tables(1.0, None, conf)
    assert float(T[0, 0, 0]) == 1.0
    k2 = sum(np.meshgrid(*[k.astype(np.float64)**2 for k in co.kvec], indexing="ij"))
    band = np.where(k2 > 0, np.exp(-0.25 / np.where(k2 > 0, k2, 1) - np.where(k2 > 0, k2, 1)**2 / 16.0), 0.0)
    np.testing.assert_allclose(T.numpy(), 1 - 0.25 * band, atol=1e-6)
    s = init_potential_correction("high_k_softening", softening_strength=0.2, softening_start=0.5,
                                  softening_stop=1.0)
    Ts, _ = s.transfer_tables(1.0, None, conf)
    assert float(Ts[0, 0, 0]) == 1.0 and float(Ts.min()) < 1.0 and float(Ts.min()) >= 0.8 - 1e-6


def test_mesh_cnn_parameters_follow_haiku_layout_and_init():
    """Parameter names and shapes of MeshResidualPotentialCorrection
    (corrections/mesh_cnn.py:80-109): stem over 5 input channels, depth-1
    residual blocks, a zero-initialised output layer and a gain of stddev
    output_init_scale; the window+mesh-CNN model combines both."""
    from pmpp_b200.corrections import CombinedPotentialCorrection, init_potential_correction
    c = init_potential_correction("mesh_cnn", mesh_channels=8, mesh_depth=4, output_init_scale=0.05, device="cpu")
    shapes = dict(c.layout)
    assert shapes["stem/w"] == (3, 3, 3, 5, 8) and shapes["out/w"] == (3, 3, 3, 8, 1)
    assert [n for n in shapes if n.startswith("block_")] == [f"block_{i}_conv{j}/{p}" for i in range(3)
                                                              for j in (1, 2) for p in ("w", "b")]
    assert float(c.view("out/w").abs().max()) == 0.0 and float(c.view("stem/b").abs().max()) == 0.0
    w = c.view("stem/w")
    assert abs(float(w.std()) - (1 / 135)**0.5) < 0.03 and float(w.abs().max()) <= 2 * (1 / 135)**0.5 / 0.8796 + 1e-6
    assert float(c.view("direct_gain/w").abs().max()) < 0.5
    cw = init_potential_correction("pm_window+mesh_cnn", channels=4, depth=2, device="cpu")
    assert isinstance(cw, CombinedPotentialCorrection) and cw.green_kernel == 1 and cw.mesh_cnn_part is not None
    with pytest.raises(ValueError, match="4, 8 or 16"):
        init_potential_correction("cnn", channels=6, device="cpu")


def test_oracle_mesh_cnn_reference_properties():
    """The restatement: zero output layer and zero gain give no residual, a
    zero output layer alone a uniform rescaling of the potential, and zero
    parameters leave the force unchanged."""
    from pmpp_b200.meshcnn import param_layout
    rng = np.random.default_rng(0)
    P = {n: rng.normal(size=s) * 0.2 for n, s in param_layout(4, 2)}
    P["out/w"][:] = 0
    P["out/b"][:] = 0
    S, phi = rng.normal(size=(6, 6, 6)), rng.normal(size=(6, 6, 6))
    R = opm.mesh_cnn_residual(P, S, phi, 1.0, 0.3, 0.8, depth=2, max_residual=0.2)
    np.testing.assert_allclose(R / phi, (R / phi).flat[0], rtol=1e-12)
    P["direct_gain/w"][:] = 0
    P["direct_gain/b"][:] = 0
    assert np.all(opm.mesh_cnn_residual(P, S, phi, 1.0, 0.3, 0.8, depth=2, max_residual=0.2) == 0)
    co = opm.Conf(4.0, (4, 4, 4), mesh_shape=2)
    pmid, disp = opm.gen_grid(co)
    disp = disp + rng.normal(0, 1.0, disp.shape)
    np.testing.assert_allclose(opm.gravity_cnn(pmid, disp, co, 0.3, P, 1.0, 0.8, depth=2),
                               opm.gravity(pmid, disp, co, 0.3), rtol=1e-12, atol=1e-14)


def test_float64_transfers_match_oracle():
    """The float64 build's window, PGD and softening tables are float64 and
    match the oracle's float64 restatements to rounding."""
    import pmpp_b200 as pb
    from pmpp_b200.corrections import init_potential_correction
    conf = pb.Configuration(4.0, (16, 16, 16), 2, float_dtype="float64", device="cpu")
    co = opm.Conf(4.0, (16, 16, 16), mesh_shape=2, float_dtype=np.float64)
    pgd = dict(alpha0=0.3, A=0.4, B=0.1, kl=0.1, ks=1.0)
    cases = [("pm_window", opm.window_gain(co)), ("pgd", opm.pgd_transfer(co, 0.5, **pgd)),
             ("softening", opm.softening_transfer(co, 0.6, 0.5, 1.0))]
    for model, ref in cases:
        T, R = init_potential_correction(model, strength=0.6, start=0.5, **pgd).transfer_tables(0.5, None, conf)
        assert R is None and T.dtype == torch.float64, model
        np.testing.assert_allclose(T.numpy(), ref, rtol=1e-13, atol=1e-15, err_msg=model)


def test_float64_correction_tables_route_and_refuse():
    """x64.correction_tables: float64 spectral tables (the discrete-Laplacian
    wavenumbers and FastPM's derivative when asked for), the float64 transfer
    and the interlacing flag; the mesh CNN, a learned radial transfer and a
    float32 transfer are refused."""
    import pmpp_b200 as pb
    from pmpp_b200 import x64
    from pmpp_b200.corrections import init_potential_correction
    conf = pb.Configuration(4.0, (8, 8, 8), 2, float_dtype="float64", device="cpu")
    t0, T0, il0 = x64.correction_tables(conf, "cpu")
    assert t0.dtype == torch.float64 and T0 is None and not il0
    t, T, il = x64.correction_tables(conf, "cpu", init_potential_correction("fastpm_3_4"), 0.5)
    assert T is None and not il and t.dtype == torch.float64
    assert torch.equal(t, conf.spectral_tables("mesh", "cpu", 1, 1)) and not torch.equal(t, t0)
    t, T, il = x64.correction_tables(conf, "cpu", init_potential_correction("windowed_pgd", interlacing=True), 0.5)
    assert il and T.dtype == torch.float64 and T.shape == (16, 16, 9)

    class Radial:
        green_kernel = 0

        def transfer_tables(self, a, cosmo, conf):
            return None, torch.ones(10, dtype=torch.float32)

    class Float32Transfer(Radial):
        def transfer_tables(self, a, cosmo, conf):
            return torch.ones((16, 16, 9), dtype=torch.float32), None

    class Cnn(Radial):
        mesh_cnn = True

    with pytest.raises(NotImplementedError):
        x64.correction_tables(conf, "cpu", Radial(), 0.5)
    with pytest.raises(NotImplementedError):
        x64.correction_tables(conf, "cpu", Cnn(), 0.5)
    with pytest.raises(TypeError):
        x64.correction_tables(conf, "cpu", Float32Transfer(), 0.5)
