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
