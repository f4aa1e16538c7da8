"""Mesh-CNN residual potential correction (corrections/mesh_cnn.py:66-265,
corrections/core.py:321-331) on the GPU against the float64 restatement in
oracle/pm.py (mesh_cnn_residual, gravity_cnn).

Cases (after the reference's tests/test_potential_correction.py:81-126):
identity at init with output_init_scale 0; a pure global rescaling of the
potential at init (the output convolution starts at zero); with random
parameters, the residual within 1e-5 of the oracle (relative to its maximum)
and every cotangent of the hand-written backward -- source, potential,
parameters, conditioning features -- within 1e-4 of the oracle's
fourth-order directional differences (float32 kernels against a smooth
float64 function); the corrected force within 1e-5 of the oracle and its
adjoint (positions, parameters, Omega_m) within 2e-4 of directional
differences of the oracle force; a short run's reverse sweep equal to the
per-operation adjoints stepped by hand.
"""
import numpy as np
import pytest
import torch

from oracle import pm as opm
from tests.helpers import random_particles, rel_err

pytestmark = pytest.mark.gpu


def _cnn(channels=4, depth=3, max_residual=0.2, scale=0.3, seed=0, **kw):
    from pmpp_b200.meshcnn import MeshCNNCorrection
    c = MeshCNNCorrection(channels=channels, depth=depth, max_residual=max_residual, seed=seed, **kw)
    if scale:
        g = torch.Generator().manual_seed(seed + 100)
        c.params += (scale * torch.randn(c.params.shape, generator=g)).cuda() * (c.params == 0)
    return c


def _fields(shape=(16, 16, 16), seed=1):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=shape)
    # smooth-ish fields: a few Fourier modes plus noise
    k = np.fft.rfftn(x)
    S = np.fft.irfftn(k * np.exp(-0.05 * np.arange(k.shape[2])), s=shape)
    phi = np.fft.irfftn(np.fft.rfftn(rng.normal(size=shape)) / (1 + np.arange(k.shape[2])), s=shape)
    return S.astype(np.float32), phi.astype(np.float32)


def _fd(f, eps):
    return (-f(2 * eps) + 8 * f(eps) - 8 * f(-eps) + f(-2 * eps)) / (12 * eps)


def test_identity_and_global_rescaling_at_init():
    from pmpp_b200.meshcnn import MeshCNNCorrection
    S, phi = _fields((8, 8, 8))
    St, pt = torch.from_numpy(S).cuda(), torch.from_numpy(phi).cuda()
    c0 = MeshCNNCorrection(channels=4, depth=2, max_residual=0.2, output_init_scale=0.0, allow_missing_sigma8=True)
    R0 = c0.residual(St, pt, 1.0, None).cpu().numpy()
    assert np.all(R0 == 0.0)
    c1 = MeshCNNCorrection(channels=4, depth=2, max_residual=0.2, output_init_scale=1e-2, seed=1,
                           allow_missing_sigma8=True)
    ratio = c1.residual(St, pt, 1.0, None).cpu().numpy() / phi
    np.testing.assert_allclose(ratio, np.full_like(ratio, ratio.flat[0]), atol=1e-6, rtol=1e-6)
    assert abs(ratio.flat[0]) > 0


@pytest.mark.parametrize("channels,depth", [(4, 3), (8, 2)])
def test_residual_and_backward_match_oracle(channels, depth):
    import pmpp_b200 as pb
    cnn = _cnn(channels, depth, seed=3)
    S, phi = _fields((16, 12, 20), seed=4)
    conf = pb.Configuration(2.0, (8, 6, 10), 2, device="cuda")
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    a = 0.6
    f = cnn.features(a, cos)
    St, pt = torch.from_numpy(S).cuda(), torch.from_numpy(phi).cuda()
    R = cnn.residual(St, pt, a, cos).cpu().numpy()
    P = cnn.params_dict()
    Rref = opm.mesh_cnn_residual(P, S.astype(np.float64), phi.astype(np.float64), *f, depth=depth, max_residual=0.2)
    assert rel_err(R, Rref) < 1e-5
    rng = np.random.default_rng(6)
    Rc = rng.normal(size=S.shape).astype(np.float32)
    dS, dphi, dpar, dfeat = cnn.residual_adjoint(torch.from_numpy(Rc).cuda())
    dS, dphi, dpar = dS.cpu().numpy(), dphi.cpu().numpy(), dpar.cpu().numpy()
    vS, vp = rng.normal(size=S.shape), rng.normal(size=S.shape)
    L = lambda S_, p_, par=P, ff=f: float((opm.mesh_cnn_residual(par, S_, p_, *ff, depth=depth, max_residual=0.2)
                                          * Rc).sum())
    S64, p64 = S.astype(np.float64), phi.astype(np.float64)
    fd_S = _fd(lambda t: L(S64 + t * vS, p64), 1e-3)
    fd_p = _fd(lambda t: L(S64, p64 + t * vp), 1e-3)
    np.testing.assert_allclose((dS * vS).sum(), fd_S, rtol=1e-4)
    np.testing.assert_allclose((dphi * vp).sum(), fd_p, rtol=1e-4)
    # parameters: one random direction over the whole flat vector
    names = [n for n, _ in cnn.layout]
    vpar = {n: rng.normal(size=P[n].shape) for n in names}
    fd_par = _fd(lambda t: L(S64, p64, {n: P[n] + t * vpar[n] for n in names}), 1e-3)
    flat_v = np.concatenate([vpar[n].ravel() for n in names])
    np.testing.assert_allclose((dpar * flat_v).sum(), fd_par, rtol=1e-4)
    # conditioning features (a, Omega_m, sigma8)
    for k in range(3):
        e = np.eye(3)[k]
        fd_f = _fd(lambda t: L(S64, p64, P, list(np.asarray(f) + t * e)), 1e-3)
        np.testing.assert_allclose(dfeat[k], fd_f, rtol=1e-4, atol=1e-6 * abs(fd_S))


def test_force_with_mesh_cnn_and_adjoint():
    import pmpp_b200 as pb
    from pmpp_b200.gravity import force, force_vjp
    co = opm.Conf(4.0, (8, 8, 8), mesh_shape=2, a_start=0.1)
    conf = pb.Configuration(4.0, (8, 8, 8), 2, a_start=0.1, device="cuda")
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    cnn = _cnn(4, 2, scale=0.3, seed=5)
    P = cnn.params_dict()
    a = 0.5
    s8 = cnn.features(a, cos)[2]
    pmid, disp = random_particles(co, 9, 1.5)
    pm, d = torch.from_numpy(pmid).cuda(), torch.from_numpy(disp).cuda()
    om = cos.Omega_m
    acc, F = force(pm, d.clone(), conf, om, a=a, cosmo=cos, correction=cnn)
    kern = opm.potential_kernel(co)
    ref = opm.gravity_cnn(pmid, disp, co, om, P, a, s8, kern, depth=2, max_residual=0.2)
    assert rel_err(acc.cpu().numpy(), ref) < 1e-5
    # the residual changes the force (the test is not vacuous)
    assert rel_err(ref, opm.gravity(pmid, disp, co, om)) > 1e-3
    rng = np.random.default_rng(11)
    ac = rng.normal(size=disp.shape).astype(np.float32)
    cnn.zero_grad()
    om_out = []
    dc = force_vjp(pm, d, conf, om, F, torch.from_numpy(ac).cuda(), a=a, cosmo=cos, correction=cnn,
                   om_out=om_out).cpu().numpy()
    # oracle in float64 positions for the differences
    co64 = opm.Conf(4.0, (8, 8, 8), mesh_shape=2, a_start=0.1, float_dtype=np.float64)
    kern64 = opm.potential_kernel(co64)
    d64 = disp.astype(np.float64)
    Lf = lambda dd, par=P, o=om: float((opm.gravity_cnn(pmid, dd, co64, o, par, a, s8, kern64, depth=2,
                                                        max_residual=0.2) * ac).sum())
    v = rng.normal(size=disp.shape)
    v /= np.linalg.norm(v)
    np.testing.assert_allclose((dc * v).sum(), _fd(lambda t: Lf(d64 + t * v), 1e-4), rtol=2e-4)
    names = [n for n, _ in cnn.layout]
    vpar = {n: rng.normal(size=P[n].shape) for n in names}
    fd_par = _fd(lambda t: Lf(d64, {n: P[n] + t * vpar[n] for n in names}), 1e-3)
    flat_v = np.concatenate([vpar[n].ravel() for n in names])
    np.testing.assert_allclose((cnn.grad.cpu().numpy() * flat_v).sum(), fd_par, rtol=2e-4)
    np.testing.assert_allclose(om_out[0], _fd(lambda t: Lf(d64, P, om + t), 1e-4), rtol=2e-4)


def test_reverse_sweep_with_mesh_cnn_matches_per_operation_adjoints():
    import pmpp_b200 as pb
    a = np.linspace(0.1, 0.7, 3)
    co = opm.Conf(4.0, (16, 16, 16), mesh_shape=2, a_start=0.1, a_custom=a)
    conf = pb.Configuration(4.0, (16, 16, 16), 2, a_start=0.1, a_custom=a, device="cuda")
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    corr = pb.corrections.CombinedPotentialCorrection(window=pb.corrections.PMWindowCompensation(),
                                                      mesh_cnn=_cnn(4, 2, seed=7))
    pmid, disp = random_particles(co, 12, 1.0)
    vel = np.random.default_rng(13).normal(0, 0.3, disp.shape).astype(np.float32)
    ptcl = pb.Particles(conf, torch.from_numpy(pmid).cuda(), torch.from_numpy(disp).cuda(),
                        torch.from_numpy(vel).cuda())
    run = pb.NBodyRun(conf, cos, corr)
    out = run.forward(ptcl)
    rng = np.random.default_rng(14)
    cot = pb.Particles(conf, ptcl.pmid, torch.from_numpy(rng.normal(size=disp.shape).astype(np.float32)).cuda(),
                       torch.from_numpy(rng.normal(size=disp.shape).astype(np.float32)).cuda(),
                       torch.zeros_like(out.disp))
    p_f, c_f, om_f = run.adjoint(out, cot)
    p, c, omi = out, cot, 0.0
    for a_prev, a_next in list(zip(a[:-1], a[1:]))[::-1]:
        p, c, omi, _ = pb.integrate_adj(a_prev, a_next, p, c, cos, omi, conf, corr)
    p, c, om_i, _ = pb.force_adj(float(a[0]), p, c, cos, conf, corr)
    omi += om_i
    assert rel_err(c.disp.cpu().numpy(), c_f.disp.cpu().numpy()) < 1e-5
    assert rel_err(c.vel.cpu().numpy(), c_f.vel.cpu().numpy()) < 1e-5
    np.testing.assert_allclose(omi, om_f, rtol=1e-5)
