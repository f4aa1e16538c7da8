"""GPU parity of the initial conditions, 2LPT (+ adjoint) and P(k) (+ loss gradient).

Bars: white-noise hashes bit-exact and the Gaussian modes within float32
round-off of the oracle; shared low-k modes bitwise equal across resolutions
(reference tests/test_nested_white_noise.py:53-68); linear modes, LPT states
and P(k) within 1e-5; shell mode counts exact; adjoints within 2e-3 of
float64 central differences of the oracle.
"""
import numpy as np
import pytest
import torch

from oracle import cosmology as ocos
from oracle import pm as opm
from tests.helpers import rel_err

pytestmark = pytest.mark.gpu


def _pair(shape=(16, 16, 16), mesh=2, spacing=8.0, dtype=np.float32, **kw):
    import pmpp_b200 as pb
    co = opm.Conf(spacing, shape, mesh_shape=mesh, a_start=0.1, float_dtype=dtype, **kw)
    c = pb.Configuration(spacing, shape, mesh, a_start=0.1, device="cuda", **kw)
    return pb, co, c


@pytest.mark.parametrize("shape", [(16, 16, 16), (12, 10, 8), (9, 8, 7)])
def test_white_noise_hashes_and_modes(shape):
    pb, co, conf = _pair(shape)
    from pmpp_b200 import modes as pm
    w, h = pm.white_noise_nested(1234, conf, return_hashes=True)
    ref = opm.white_noise_nested(1234, co)
    # hashes: recompute the canonical hash inputs with the oracle
    n0, n1, n2 = shape
    md = lambda n: np.where(np.arange(n) < (n + 1) // 2, np.arange(n), np.arange(n) - n)
    kx, ky, kz = np.meshgrid(md(n0), md(n1), np.arange(n2 // 2 + 1), indexing="ij")
    hh = h.cpu().numpy().view(np.uint32)
    plane = (kz == 0) | ((n2 % 2 == 0) & (kz == n2 // 2))
    sel = ~plane
    hr = opm.hash_mode(1234, kx[sel], ky[sel], kz[sel], 0xA24BAED4)
    assert np.array_equal(hh[..., 0][sel], hr)
    got = w.cpu().numpy()
    assert np.abs(got - ref).max() < 5e-6 * np.abs(ref).max()


def test_nested_noise_shared_low_k_modes_bitwise():
    from pmpp_b200 import modes as pm
    pb, co32, c32 = _pair((32, 32, 32), spacing=8.0)
    _, co64, c64 = _pair((64, 64, 64), spacing=4.0)
    a = pm.white_noise_nested(7, c32).cpu().numpy()
    b = pm.white_noise_nested(7, c64).cpu().numpy()
    k = 8
    ix = np.r_[0:k, -k + 1:0]
    sa = a[np.ix_(ix % 32, ix % 32, np.arange(1, k))]
    sb = b[np.ix_(ix % 64, ix % 64, np.arange(1, k))]
    assert np.array_equal(sa.view(np.uint32), sb.view(np.uint32))


def test_linear_modes_matches_oracle():
    pb, co, conf = _pair()
    from pmpp_b200 import modes as pm
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    oc = opm.boltzmann(ocos.Cosmo(), co)
    w = pm.white_noise_nested(3, conf)
    lm = pm.linear_modes(w, cos, conf).cpu().numpy()
    ref = opm.linear_modes(w.cpu().numpy(), oc, co)
    assert np.abs(lm - ref).max() < 1e-5 * np.abs(ref).max()


@pytest.mark.parametrize("order", [1, 2])
def test_lpt_matches_oracle(order):
    pb, co, conf = _pair(lpt_order=order)
    from pmpp_b200 import lpt as pl, modes as pm
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    oc = opm.boltzmann(ocos.Cosmo(), co)
    lm = pm.linear_modes(pm.white_noise_nested(5, conf), cos, conf)
    ptcl = pl.lpt(lm, cos, conf)
    pmid, disp, vel = opm.lpt(lm.cpu().numpy(), oc, co)
    assert np.array_equal(ptcl.pmid.cpu().numpy(), pmid)
    assert rel_err(ptcl.disp.cpu().numpy(), disp) < 1e-5
    assert rel_err(ptcl.vel.cpu().numpy(), vel) < 1e-5


def test_lpt_adjoint_vs_finite_differences():
    pb, co, conf = _pair((8, 8, 8), spacing=16.0)
    _, co64, _ = _pair((8, 8, 8), spacing=16.0, dtype=np.float64)
    from pmpp_b200 import lpt as pl, modes as pm
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    oc = opm.boltzmann(ocos.Cosmo(), co64)
    lm = pm.linear_modes(pm.white_noise_nested(9, conf), cos, conf)
    res = pl.lpt_full(lm, cos, conf)
    rng = np.random.default_rng(0)
    dc = rng.normal(size=(512, 3)).astype(np.float32)
    vc = rng.normal(size=(512, 3)).astype(np.float32)
    mc, _ = pl.lpt_vjp(res, torch.from_numpy(dc).cuda(), torch.from_numpy(vc).cuda(), cos, conf)
    mc = mc.cpu().numpy()
    base = lm.cpu().numpy().astype(np.complex128)
    # perturb interior modes only (0 < kz < Nyquist): unambiguous real/imag parts
    direction = np.zeros_like(base)
    direction[:, :, 1:-1] = rng.normal(size=direction[:, :, 1:-1].shape) + 1j * rng.normal(
        size=direction[:, :, 1:-1].shape)
    direction *= np.abs(base).mean()

    def L(m):
        _, d, v = opm.lpt(m, oc, co64)
        return float((d * dc).sum() + (v * vc).sum())

    eps = 1e-3
    fd = (L(base + eps * direction) - L(base - eps * direction)) / (2 * eps)
    ad = float((mc.real * direction.real + mc.imag * direction.imag).sum())
    np.testing.assert_allclose(ad, fd, rtol=2e-3)


def test_shell_statistics_and_pk_match_oracle():
    pb, co, conf = _pair((16, 16, 16), mesh=2)
    from pmpp_b200 import power_spectrum as ps
    k, n = ps.shell_statistics(conf)
    rk, rn = opm.shell_statistics(co.mesh_shape, co.cell_size)
    ns = ps.num_shells(conf) - 1
    assert np.array_equal(n[:ns], rn[:ns])
    np.testing.assert_allclose(k[:ns], rk[:ns], rtol=1e-12)
    rng = np.random.default_rng(1)
    rho = (1 + 0.3 * rng.normal(size=co.mesh_shape)).astype(np.float32)
    kk, pk, nm = ps.density_to_pk(torch.from_numpy(rho).cuda(), conf)
    rk2, rpk, rnm = opm.density_to_pk(rho.astype(np.float64), co)
    assert np.array_equal(nm, rnm)
    assert rel_err(pk, rpk) < 1e-5


def test_pk_loss_gradient_vs_finite_differences():
    pb, co, conf = _pair((8, 8, 8), mesh=2, spacing=16.0)
    _, co64, _ = _pair((8, 8, 8), mesh=2, spacing=16.0, dtype=np.float64)
    from pmpp_b200 import power_spectrum as ps
    rng = np.random.default_rng(2)
    pmid, disp = opm.gen_grid(co)
    disp = (disp + rng.normal(0, 3.0, size=disp.shape)).astype(np.float32)
    ptcl = pb.Particles(conf, torch.from_numpy(pmid).cuda(), torch.from_numpy(disp).cuda())
    k, pk, nm = ps.particles_to_pk(ptcl, conf)
    target = pk * np.exp(0.1 * rng.normal(size=pk.shape))
    loss, g = ps.pk_loss(ptcl, conf, target)
    g = g.cpu().numpy()

    def L(d):
        _, p, n = opm.density_to_pk(opm.scatter(pmid, d, co64), co64)
        v = (n > 0) & (p > 0)
        lr = np.log(p[v] / target[v])
        return float((lr**2).sum() / v.sum())

    np.testing.assert_allclose(loss, L(disp.astype(np.float64)), rtol=1e-4)
    direction = rng.normal(size=disp.shape)
    # CIC is piecewise linear: keep the step far below the distance at which
    # a particle crosses a cell boundary
    eps = 1e-5
    d64 = disp.astype(np.float64)
    fd = (L(d64 + eps * direction) - L(d64 - eps * direction)) / (2 * eps)
    np.testing.assert_allclose(float((g * direction).sum()), fd, rtol=2e-3)
