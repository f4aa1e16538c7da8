"""Learned Green's-function correction on the GPU.

MLP table and its backward kernel against a float64 NumPy restatement with
the same bf16-rounded weights; the transfer cotangent of the force adjoint
and the N-body parameter gradient against float64 central differences of the
oracle.
"""
import numpy as np
import pytest
import torch

from oracle import cosmology as ocos
from oracle import pm as opm
from tests.helpers import random_particles

pytestmark = pytest.mark.gpu


def _model(seed=0, scale=0.3):
    from pmpp_b200.corrections import LearnedGreen
    m = LearnedGreen("cuda", seed=seed)
    # non-trivial output layer so T != 1
    g = torch.Generator().manual_seed(seed + 1)
    m.w[-64:] = (torch.randn(64, generator=g) * scale / 8).cuda()
    m.b[-1] = 0.01
    m._sync_bf16()
    return m


def _np_params(m):
    return opm.bf16_round(m.w.cpu().numpy()), m.b.cpu().numpy().astype(np.float64)


def test_mlp_table_matches_numpy():
    import pmpp_b200 as pb
    m = _model()
    conf = pb.Configuration(8.0, (16, 16, 16), 2, device="cuda")
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    T = m.table(0.5, cos, conf).cpu().numpy()
    w, b = _np_params(m)
    ref = opm.mlp_table(w, b, 2.0 / 32, 0.5, 0.3, m._cond(0.5, cos, conf)[3], len(T))
    np.testing.assert_allclose(T, ref, rtol=2e-5, atol=2e-6)
    assert T[0] == 1.0


def test_mlp_backward_matches_finite_differences():
    import pmpp_b200 as pb
    m = _model(3)
    conf = pb.Configuration(8.0, (8, 8, 8), 2, device="cuda")
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    from pmpp_b200.corrections import radial_table_len
    L = radial_table_len(conf)
    rng = np.random.default_rng(0)
    tc = rng.normal(size=L)
    m.zero_grad()
    m.accumulate(0.4, cos, conf, torch.from_numpy(tc).cuda())
    g = m.grad.cpu().numpy().astype(np.float64)
    w, b = _np_params(m)
    s8 = m._cond(0.4, cos, conf)[3]
    p = np.concatenate([w, b])
    u = rng.normal(size=p.shape)
    nw = len(w)
    f = lambda q: float((opm.mlp_table(q[:nw], q[nw:], 2.0 / 16, 0.4, 0.3, s8, L) * tc).sum())
    eps = 1e-5
    fd = (f(p + eps * u) - f(p - eps * u)) / (2 * eps)
    np.testing.assert_allclose(float(g @ u), fd, rtol=2e-4)


def test_transfer_cotangent_matches_finite_differences():
    import pmpp_b200 as pb
    from pmpp_b200.corrections import radial_table_len
    from pmpp_b200.gravity import force, force_vjp
    co64 = opm.Conf(4.0, (8, 8, 8), mesh_shape=2, float_dtype=np.float64)
    co = opm.Conf(4.0, (8, 8, 8), mesh_shape=2)
    conf = pb.Configuration(4.0, (8, 8, 8), 2, device="cuda")
    pmid, disp = random_particles(co, seed=4, spread=2.0)
    L = radial_table_len(conf)
    rng = np.random.default_rng(1)
    table = (1 + 0.2 * rng.normal(size=L)).astype(np.float32)
    table[0] = 1
    ac = rng.normal(size=disp.shape).astype(np.float32)

    class Fixed:
        green_kernel = 0

        def transfer_tables(self, a, cosmo, conf):
            return None, torch.from_numpy(table).cuda()

    corr = Fixed()
    P = torch.from_numpy(pmid).cuda()
    D = torch.from_numpy(disp).cuda()
    nx, ny, nz = conf.mesh_shape
    S = torch.empty((nx, ny, nz // 2 + 1), dtype=torch.complex64, device="cuda")
    acc, F = force(P, D.clone(), conf, 0.3, correction=corr, src_hat_out=S)
    tc = torch.zeros(L, dtype=torch.float64, device="cuda")
    force_vjp(P, D, conf, 0.3, F, torch.from_numpy(ac).cuda(), correction=corr, src_hat=S, transfer_cot_out=tc)
    tc = tc.cpu().numpy()

    def Lf(t):
        k = opm.potential_kernel(co64, transfer=opm.radial_transfer(t, co64))
        return float((opm.gravity(pmid, disp, co64, 0.3, kernel=k) * ac).sum())

    u = rng.normal(size=L)
    u[0] = 0
    eps = 1e-4
    fd = (Lf(table + eps * u) - Lf(table - eps * u)) / (2 * eps)
    np.testing.assert_allclose(float(tc @ u), fd, rtol=1e-3)


def test_nbody_parameter_gradient_matches_finite_differences():
    import pmpp_b200 as pb
    a = np.linspace(0.1, 1.0, 3)
    co64 = opm.Conf(8.0, (8, 8, 8), mesh_shape=2, float_dtype=np.float64, a_start=0.1, a_custom=a)
    co = opm.Conf(8.0, (8, 8, 8), mesh_shape=2, a_start=0.1, a_custom=a)
    conf = pb.Configuration(8.0, (8, 8, 8), 2, a_start=0.1, a_custom=a, device="cuda")
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    oc = opm.boltzmann(ocos.Cosmo(), co64)
    m = _model(5)
    pmid, disp = random_particles(co, seed=8, spread=1.0)
    vel = np.random.default_rng(2).normal(0, 0.5, size=disp.shape).astype(np.float32)
    ptcl = pb.Particles(conf, torch.from_numpy(pmid).cuda(), torch.from_numpy(disp).cuda(),
                        torch.from_numpy(vel).cuda())
    run = pb.NBodyRun(conf, cos, correction=m)
    out = run.forward(ptcl)
    rng = np.random.default_rng(3)
    dcot = rng.normal(size=disp.shape).astype(np.float32)
    cot = pb.Particles(conf, ptcl.pmid, torch.from_numpy(dcot).cuda(), torch.zeros_like(out.disp),
                       torch.zeros_like(out.disp))
    m.zero_grad()
    run.adjoint(out, cot)
    g = m.grad.cpu().numpy().astype(np.float64)
    w, b = _np_params(m)
    nw = len(w)
    s8 = m._cond(0.1, cos, conf)[3]
    L = (8)**2 * 3 + 1

    def Lf(p):
        kern = lambda aa: opm.potential_kernel(co64, transfer=opm.radial_transfer(
            opm.mlp_table(p[:nw], p[nw:], 2.0 / 16, float(np.float32(aa)), 0.3, s8, L), co64))
        d, _, _ = opm.nbody(pmid, disp, vel, co64, oc, kernel=kern)
        return float((d * dcot).sum())

    p = np.concatenate([w, b])
    u = rng.normal(size=p.shape) * 0.01
    eps = 1e-4
    fd = (Lf(p + eps * u) - Lf(p - eps * u)) / (2 * eps)
    np.testing.assert_allclose(float(g @ u), fd, rtol=5e-3)
