"""Pin the CPU oracle against the reference's own known-answer tests.

The reference (JAX) cannot run here, so the oracle is checked against the
closed-form / invariant assertions of the reference test suite, restated:
  * tests/test_deep_gravity_spectral.py:31-63   Poisson symbols, zero mode
  * tests/test_deep_gravity_spectral.py:66-89   Nyquist-zeroed spectral gradient
  * tests/test_deep_gravity_spectral.py:253-275 uniform lattice => zero force
  * tests/test_power_spectrum.py:69-92          cross-correlation r = +-1
  * tests/test_deep_lpt_orders.py:18-66         2LPT source symmetric/bilinear,
                                                order 0 is the identity
  * tests/test_nested_white_noise.py:53-68      shared low-k modes bitwise
  * tests/test_deep_boltzmann_contracts.py:20-31 transfer normalisation
  * tests/test_finite_diff.py:87-124            adjoints vs 4th-order central
                                                differences in float64
  * tests/test_gravity_particle_nyquist_filter.py:11-40  refined force meshes do
                                                not alias the particle lattice
"""
import numpy as np
import pytest

from oracle import cosmology as ocos
from oracle import pm as opm


def _conf(shape=(4, 4, 4), dtype=np.float32, **kw):
    return opm.Conf(1.25, shape, mesh_shape=1, float_dtype=dtype, **kw)


def test_poisson_symbols_closed_form():
    conf = _conf()
    k2 = opm.k_squared(conf.kvec, np.float32)
    k2d = opm.discrete_k_squared(conf.kvec, conf.cell_size, np.float32)
    assert k2[0, 0, 0] == 0 and k2d[0, 0, 0] == 0
    assert np.all(k2d <= k2 + 2e-6)
    assert np.any(k2d < k2 - 1e-5)
    G = opm.green(conf)
    src = (np.arange(k2.size, dtype=np.float32).reshape(k2.shape) + 1).astype(np.complex64)
    expected = np.where(k2 != 0, -src / np.where(k2 == 0, 1, k2), 0)
    np.testing.assert_allclose(src * G, expected, rtol=2e-6)
    assert np.all(np.isfinite(opm.green(conf, "discrete_laplacian")))


def test_spectral_gradient_zeroes_nyquist():
    conf = _conf()
    k = np.asarray([0, np.pi / (2 * conf.cell_size), np.pi / conf.cell_size], dtype=np.float32)
    c = conf._neg_k(k)
    pot = np.asarray([1 + 2j, 2 - 1j, 3 + 4j], dtype=np.complex64)
    np.testing.assert_allclose((1j * c * pot)[:2], (-1j * k * pot)[:2], rtol=2e-6)
    assert (1j * c * pot)[2] == 0


def test_uniform_lattice_has_zero_force_and_tiny_kick_conserves_momentum():
    conf = _conf()
    pmid, disp = opm.gen_grid(conf)
    acc = opm.gravity(pmid, disp, conf, 0.3)
    np.testing.assert_allclose(acc, 0, atol=3e-7)
    disp2 = disp.copy()
    disp2[0, 0] = np.float32(1e-3)
    acc2 = opm.gravity(pmid, disp2, conf, 0.3)
    assert np.linalg.norm(acc2) > 1e-7
    assert np.linalg.norm(acc2.sum(axis=0)) < 2e-5


def test_cross_correlation_identity_and_sign():
    n = 16
    conf = opm.Conf(25.0 / n, (n, n, n), mesh_shape=1)
    rng = np.random.default_rng(4)
    d = rng.normal(size=(n, n, n))
    d -= d.mean()
    _, r, px, pa, pb, _ = opm.delta_to_cross_correlation(d, d, conf)
    np.testing.assert_allclose(r, 1.0, atol=2e-6)
    np.testing.assert_allclose(px, pa, rtol=1e-6)
    _, r2, px2, pa2, _, _ = opm.delta_to_cross_correlation(d, -d, conf)
    np.testing.assert_allclose(r2, -1.0, atol=2e-6)
    np.testing.assert_allclose(px2, -pa2, rtol=1e-6)


def test_lpt_source_symmetric_bilinear_and_diagonal_strain():
    conf = opm.Conf(1.0, (4, 4, 4), float_dtype=np.float64)
    ax = np.arange(4.0)
    x, y, z = np.meshgrid(ax, ax, ax, indexing="ij")
    ra = np.sin(2 * np.pi * x / 4) + 0.3 * np.cos(2 * np.pi * (y + z) / 4) + 0.17 * np.sin(2 * np.pi * (x + y) / 4)
    rb = 0.4 * np.cos(2 * np.pi * y / 4) - 0.21 * np.sin(2 * np.pi * (x + z) / 4)
    pa, pb = np.fft.rfftn(ra), np.fft.rfftn(rb)
    ab = opm.lpt_source(pa, conf, pb)
    ba = opm.lpt_source(pb, conf, pa)
    np.testing.assert_allclose(ab, ba, rtol=2e-14, atol=2e-14)
    eps = 1e-5
    fd = (opm.lpt_source(pa + eps * pb, conf) - opm.lpt_source(pa - eps * pb, conf)) / (2 * eps)
    np.testing.assert_allclose(fd, 2 * ab, rtol=2e-10, atol=2e-10)


def test_lpt_order_zero_is_identity():
    conf = opm.Conf(1.0, (4, 4, 4), float_dtype=np.float64, lpt_order=0, a_start=0.1)
    cosmo = opm.boltzmann(ocos.Cosmo(), conf)
    pmid, disp, vel = opm.lpt(np.zeros((4, 4, 3), dtype=np.complex128), cosmo, conf)
    assert np.all(disp == 0) and np.all(vel == 0)


def test_nested_white_noise_shared_low_k_modes_bitwise():
    c32 = opm.Conf(8.0, (32, 32, 32))
    c64 = opm.Conf(4.0, (64, 64, 64))
    a = opm.white_noise_nested(7, c32)
    b = opm.white_noise_nested(7, c64)
    k = 15
    ix = np.r_[0:k + 1, -k:0]
    sa = a[np.ix_(ix % 32, ix % 32, np.arange(0, 16))]
    sb = b[np.ix_(ix % 64, ix % 64, np.arange(0, 16))]
    assert np.array_equal(sa.view(np.uint32), sb.view(np.uint32))


def test_white_noise_is_hermitian_consistent():
    conf = opm.Conf(1.0, (8, 6, 8))
    w = opm.white_noise_nested(3, conf).astype(np.complex128)
    full = np.fft.irfftn(w, s=conf.ptcl_grid_shape)
    np.testing.assert_allclose(np.fft.rfftn(full), w, atol=1e-12)


def test_transfer_normalisation_and_no_wiggle_monotone():
    conf = opm.Conf(1.0, (4, 4, 4))
    c = ocos.Cosmo()
    k = np.concatenate(([0.0], np.geomspace(1e-4, 0.5, 64)))
    Tb = ocos.transfer_fit(k, c)
    Ts = ocos.transfer_fit(k, c, nowiggle=True)
    assert Tb[0] == 1 and Ts[0] == 1
    np.testing.assert_allclose(Ts[1], Tb[1], rtol=2e-3, atol=2e-6)
    assert np.all(np.diff(Ts) <= 1e-12)


def _fd4(f, x, v, eps=1e-4):
    return (-f(x + 2 * eps * v) + 8 * f(x + eps * v) - 8 * f(x - eps * v) + f(x - 2 * eps * v)) / (12 * eps)


def test_oracle_adjoints_vs_finite_differences():
    conf = opm.Conf(4.0, (6, 6, 6), mesh_shape=2, float_dtype=np.float64)
    rng = np.random.default_rng(0)
    pmid, disp = opm.gen_grid(conf)
    disp = disp + rng.normal(0, 2.0, size=disp.shape)
    v = rng.normal(size=disp.shape)
    v /= np.linalg.norm(v)
    mc = rng.normal(size=conf.mesh_shape)
    dc, _ = opm.scatter_vjp(pmid, disp, conf, mc)
    fd = _fd4(lambda d: (opm.scatter(pmid, d, conf) * mc).sum(), disp, v)
    np.testing.assert_allclose((dc * v).sum(), fd, rtol=1e-7, atol=1e-9)
    mesh = rng.normal(size=(3, ) + conf.mesh_shape)
    vc = rng.normal(size=disp.shape)
    dc, mco = opm.gather_vjp(pmid, disp, conf, mesh, vc)
    fd = _fd4(lambda d: (opm.gather(pmid, d, conf, mesh) * vc).sum(), disp, v)
    np.testing.assert_allclose((dc * v).sum(), fd, rtol=1e-7, atol=1e-9)
    u = rng.normal(size=mesh.shape)
    fd = _fd4(lambda m: (opm.gather(pmid, disp, conf, m) * vc).sum(), mesh, u)
    np.testing.assert_allclose((mco * u).sum(), fd, rtol=1e-7, atol=1e-9)
    ac = rng.normal(size=disp.shape)
    dc, om = opm.gravity_vjp(pmid, disp, conf, 0.3, ac)
    fd = _fd4(lambda d: (opm.gravity(pmid, d, conf, 0.3) * ac).sum(), disp, v)
    np.testing.assert_allclose((dc * v).sum(), fd, rtol=1e-7, atol=1e-9)


@pytest.mark.parametrize("mesh", [2, 3])
def test_oracle_interlaced_gravity_adjoint_vs_finite_differences(mesh):
    """The interlaced force (gravity.py:446-463) and its transpose, with the
    window and PGD transfers on, against 4th-order differences in float64;
    the interlaced force of a uniform lattice is zero too."""
    conf = opm.Conf(4.0, (6, 6, 6), mesh_shape=mesh, float_dtype=np.float64)
    rng = np.random.default_rng(1)
    pmid, disp = opm.gen_grid(conf)
    kern = opm.potential_kernel(conf, "discrete_laplacian", opm.window_gain(conf) * opm.pgd_transfer(conf, 0.5))
    assert np.abs(opm.gravity(pmid, disp, conf, 0.3, kern, interlacing=True)).max() < 1e-12
    disp = disp + rng.normal(0, 2.0, size=disp.shape)
    v = rng.normal(size=disp.shape)
    v /= np.linalg.norm(v)
    ac = rng.normal(size=disp.shape)
    dc, om = opm.gravity_vjp(pmid, disp, conf, 0.3, ac, kern, interlacing=True)
    fd = _fd4(lambda d: (opm.gravity(pmid, d, conf, 0.3, kern, interlacing=True) * ac).sum(), disp, v)
    np.testing.assert_allclose((dc * v).sum(), fd, rtol=1e-7, atol=1e-9)
    fdo = _fd4(lambda o: (opm.gravity(pmid, disp, conf, 0.3 + o[0], kern, interlacing=True) * ac).sum(),
               np.zeros(1), np.ones(1))
    np.testing.assert_allclose(om, fdo, rtol=1e-7)
    # interlacing changes the force (it is not the regular one)
    reg = opm.gravity(pmid, disp, conf, 0.3, kern)
    assert np.abs(opm.gravity(pmid, disp, conf, 0.3, kern, interlacing=True) - reg).max() > 1e-3 * np.abs(reg).max()


def test_oracle_nbody_adjoint_vs_finite_differences():
    conf = opm.Conf(8.0, (6, 6, 6), mesh_shape=2, float_dtype=np.float64, a_start=0.1,
                    a_custom=np.linspace(0.1, 1.0, 4))
    cosmo = opm.boltzmann(ocos.Cosmo(), conf)
    rng = np.random.default_rng(1)
    pmid, disp = opm.gen_grid(conf)
    disp = disp + rng.normal(0, 1.0, size=disp.shape)
    vel = rng.normal(0, 0.3, size=disp.shape)
    dcot = rng.normal(size=disp.shape)
    vcot = rng.normal(size=disp.shape)
    d, vv, a = opm.nbody(pmid, disp, vel, conf, cosmo)
    _, _, dc, vc, _ = opm.nbody_adj(pmid, d, vv, a, dcot, vcot, np.zeros_like(dcot), conf, cosmo, om_grads=False)
    u = rng.normal(size=disp.shape)
    u /= np.linalg.norm(u)

    def L(dd):
        o = opm.nbody(pmid, dd, vel, conf, cosmo)
        return float((o[0] * dcot).sum() + (o[1] * vcot).sum())

    np.testing.assert_allclose((dc * u).sum(), _fd4(L, disp, u, 1e-4), rtol=1e-6)


def _x_force_modes(mesh, res=16, box=1000.0, amp=0.5):
    """|rFFT| of the x-mean of the x force for lattice positions displaced by
    amp sin(2 pi x / box) along x (ordered particles: pmid the lattice cell,
    disp the nearest-image offset), normalised by res / 2."""
    conf = opm.Conf(box / res, (res, res, res), mesh_shape=mesh, a_start=1 / 128, a_nbody_maxstep=1 / 20)
    pmid, _ = opm.gen_grid(conf)
    axis = np.arange(res, dtype=np.float32) * np.float32(box / res)
    x, y, z = np.meshgrid(axis, axis, axis, indexing="ij")
    pos = np.stack([x, y, z], axis=-1).reshape(-1, 3)
    pos[:, 0] = (pos[:, 0] + np.float32(amp) * np.sin(np.float32(2 * np.pi / box) * pos[:, 0])) % np.float32(box)
    disp = pos.astype(np.float64) - pmid.astype(np.float64) * conf.cell_size
    disp = ((disp + box / 2) % box - box / 2).astype(np.float32)
    acc = opm.gravity(pmid, disp, conf, 0.3)
    mean_x = acc[:, 0].reshape(res, res, res).mean(axis=(1, 2))
    return np.abs(np.fft.rfft(mean_x)) / (res / 2)


def test_refined_force_mesh_does_not_alias_particle_lattice():
    base = _x_force_modes(1)[1]
    for mesh in (2, 4):
        modes = _x_force_modes(mesh)
        assert np.isclose(modes[1], base, rtol=0.03)
        assert modes[2] < 0.10 * base
