"""End-to-end differentiable run on the GPU against the float64 oracle.

White noise -> linear modes -> 2LPT -> KDK -> P(k); forward P(k) within 1e-3
of the oracle's float32 pipeline, and the hand-written reverse pass (noise
modes, Omega_m, A_s) within 2e-2 of float64 central differences of the
oracle pipeline (float32 chaos over the steps bounds the agreement).
"""
import numpy as np
import pytest
import torch

from oracle import cosmology as ocos
from oracle import pm as opm

pytestmark = pytest.mark.gpu

A = np.linspace(0.1, 1.0, 4)


def _setup(dtype=np.float32):
    import pmpp_b200 as pb
    co = opm.Conf(16.0, (8, 8, 8), mesh_shape=2, a_start=0.1, a_custom=A, float_dtype=dtype)
    c = pb.Configuration(16.0, (8, 8, 8), 2, a_start=0.1, a_custom=A, device="cuda")
    return pb, co, c


def _oracle_loss(omega, co, target, Om=0.3, As=2.0):
    c = opm.boltzmann(ocos.Cosmo(Omega_m=Om, A_s_1e9=As), co)
    lin = opm.linear_modes(omega, c, co)
    pmid, d, v = opm.lpt(lin, c, co)
    d2, _, _ = opm.nbody(pmid, d, v, co, c)
    _, p, n = opm.density_to_pk(opm.scatter(pmid, d2, co), co)
    lr = np.log(p / target)
    return float((lr**2).mean()), p


def test_pipeline_forward_and_gradients():
    pb, co, conf = _setup()
    _, co64, _ = _setup(np.float64)
    from pmpp_b200 import modes as pm, pipeline
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    omega = pm.white_noise_nested(11, conf)
    model = pipeline.ForwardModel(conf, cos)
    model.forward(omega)
    om64 = omega.cpu().numpy().astype(np.complex128)
    ref_loss, ref_pk = _oracle_loss(om64, co, np.ones(1))
    k, pk, n = pb.power_spectrum.particles_to_pk(model.final, conf)
    np.testing.assert_allclose(pk, ref_pk, rtol=1e-3)
    target = ref_pk * np.exp(0.2 * np.sin(np.arange(len(ref_pk))))
    loss, g = model.loss(target)
    np.testing.assert_allclose(loss, _oracle_loss(om64, co64, target)[0], rtol=1e-3)
    grads = model.backward(g)
    mc = grads["modes"].cpu().numpy()
    rng = np.random.default_rng(3)
    direction = np.zeros_like(om64)
    direction[:, :, 1:-1] = rng.normal(size=direction[:, :, 1:-1].shape) + 1j * rng.normal(
        size=direction[:, :, 1:-1].shape)
    eps = 1e-5
    fd = (_oracle_loss(om64 + eps * direction, co64, target)[0] -
          _oracle_loss(om64 - eps * direction, co64, target)[0]) / (2 * eps)
    ad = float((mc.real * direction.real + mc.imag * direction.imag).sum())
    np.testing.assert_allclose(ad, fd, rtol=2e-2)
    h = 1e-5
    fd_om = (_oracle_loss(om64, co64, target, Om=0.3 + h)[0] - _oracle_loss(om64, co64, target, Om=0.3 - h)[0]) / (2 * h)
    np.testing.assert_allclose(grads["Omega_m"], fd_om, rtol=2e-2)
    fd_as = (_oracle_loss(om64, co64, target, As=2.0 + 1e-5)[0] -
             _oracle_loss(om64, co64, target, As=2.0 - 1e-5)[0]) / 2e-5
    np.testing.assert_allclose(grads["A_s_1e9"], fd_as, rtol=2e-2)


def test_gradients_sixteen_modes_and_sigma8():
    """Reverse pass against float64 central differences of the oracle pipeline:
    16 random single white-noise coefficients, sigma8 at fixed Omega_m and
    Omega_m at fixed sigma8 (sigma8_chain); 16^3 particles / 32^3 mesh, 6 steps."""
    import pmpp_b200 as pb
    from pmpp_b200 import modes as pm, pipeline
    a = np.linspace(0.1, 1.0, 7)
    kw = dict(n_s=0.96, Omega_b=0.05, h=0.7)
    conf = pb.Configuration(4.0, (16, 16, 16), 2, a_start=0.1, a_custom=a, device="cuda")
    co64 = opm.Conf(4.0, (16, 16, 16), mesh_shape=2, a_start=0.1, a_custom=a, float_dtype=np.float64)
    cos = pb.Cosmology.from_sigma8(conf, 0.8, Omega_m=0.3, **kw)
    omega = pm.white_noise_nested(3, conf)
    model = pipeline.ForwardModel(conf, cos)
    model.forward(omega)
    _, pk0, _ = pb.power_spectrum.particles_to_pk(model.final, conf)
    target = pk0 * (1.0 + 0.1 * np.sin(np.arange(len(pk0))))
    loss, g = model.loss(target)
    grads = model.backward(g)
    d_s8, d_om = pipeline.sigma8_chain(grads, cos, conf)
    om64 = omega.cpu().numpy().astype(np.complex128)

    def oracle(w, s8=0.8, Om=0.3):
        c = opm.cosmo_from_sigma8(co64, s8, Omega_m=Om, **kw)
        lin = opm.linear_modes(w, c, co64)
        pmid, d, v = opm.lpt(lin, c, co64)
        d2, _, _ = opm.nbody(pmid, d, v, co64, c)
        _, p, _ = opm.density_to_pk(opm.scatter(pmid, d2, co64), co64)
        return float((np.log(p / target)**2).mean())

    np.testing.assert_allclose(loss, oracle(om64), rtol=2e-3)
    rng = np.random.default_rng(21)
    mc = grads["modes"].cpu().numpy()
    ad, fd = [], []
    eps = 1e-4
    for _ in range(16):
        ix, iy, iz = rng.integers(0, 16), rng.integers(0, 16), rng.integers(1, 8)
        imag = bool(rng.integers(0, 2))
        e = np.zeros_like(om64)
        e[ix, iy, iz] = 1j if imag else 1.0
        fd.append((oracle(om64 + eps * e) - oracle(om64 - eps * e)) / (2 * eps))
        ad.append(mc[ix, iy, iz].imag if imag else mc[ix, iy, iz].real)
    ad, fd = np.array(ad), np.array(fd)
    assert np.linalg.norm(ad - fd) < 3e-2 * np.linalg.norm(fd)
    h = 1e-4
    fd_s8 = (oracle(om64, s8=0.8 + h) - oracle(om64, s8=0.8 - h)) / (2 * h)
    np.testing.assert_allclose(d_s8, fd_s8, rtol=2e-2)
    fd_om = (oracle(om64, Om=0.3 + h) - oracle(om64, Om=0.3 - h)) / (2 * h)
    np.testing.assert_allclose(d_om, fd_om, rtol=3e-2)
