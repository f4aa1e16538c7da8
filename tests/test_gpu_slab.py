"""Slab-decomposed PM (pmpp_b200/slab.py) on one GPU with P ranks in one
process (LocalComm), against the single-GPU force and KDK integration.

Cases (after the reference's distributed tests, which compare the sharded run
with the single-device one): the slab force within 1e-5 of pmb_force for 2 and
4 slabs (the halo plane is summed in float, so not bit for bit); three KDK
steps with routing after every drift within 1e-5 (positions and velocities)
of nbody.integrate; every particle owned by exactly one rank after routing,
in its rank's slab; a capacity below a rank's share fails before anything
moves; the slab force adjoint within 1e-5 of force_vjp; the reverse sweep on
the slabs (cotangents routed with their particles) within 1e-5 of
nbody.integrate_adj / force_adj stepped by hand (initial positions and both
cotangents), the Omega_m cotangent within 1e-3 (a sum with cancellation).
"""
import numpy as np
import pytest
import torch

from oracle import pm as opm
from tests.helpers import random_particles, rel_err

pytestmark = pytest.mark.gpu


def _setup(shape=(32, 32, 32), mesh=2, spread=2.0, seed=3, a_custom=None):
    import pmpp_b200 as pb
    co = opm.Conf(4.0, shape, mesh_shape=mesh, a_start=0.1)
    conf = pb.Configuration(4.0, shape, mesh, a_start=0.1, a_custom=a_custom, device="cuda")
    pmid, disp = random_particles(co, seed=seed, spread=spread)
    return pb, conf, torch.from_numpy(pmid).cuda(), torch.from_numpy(disp).cuda()


def _order(conf, pmid):
    _, ny, nz = conf.mesh_shape
    p = pmid.to(torch.int64)
    return torch.argsort((p[:, 0] * ny + p[:, 1]) * nz + p[:, 2])


@pytest.mark.parametrize("P", [2, 4])
def test_slab_force_matches_single_gpu(P):
    from pmpp_b200.gravity import force
    from pmpp_b200.slab import LocalComm, SlabPM
    pb, conf, pmid, disp = _setup()
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    ref, _ = force(pmid, disp.clone(), conf, cos.Omega_m)
    ref = ref[_order(conf, pmid)]
    slab = SlabPM(conf, LocalComm(P))
    states = slab.distribute(pmid, disp)
    assert sum(s.pmid.shape[0] for s in states) == pmid.shape[0]
    slab.force(states, cos.Omega_m)
    _, _, _, acc = slab.collect(states)
    assert rel_err(acc.cpu().numpy(), ref.cpu().numpy()) < 1e-5


@pytest.mark.parametrize("P", [2, 4])
def test_slab_nbody_matches_single_gpu(P):
    from pmpp_b200.nbody import force_state, integrate
    from pmpp_b200.slab import LocalComm, SlabPM
    a = np.linspace(0.1, 0.5, 4)
    pb, conf, pmid, disp = _setup(spread=1.0, a_custom=a)
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    vel = torch.from_numpy(np.random.default_rng(4).normal(0, 3.0, disp.shape).astype(np.float32)).cuda()
    p = pb.Particles(conf, pmid, disp.clone(), vel.clone())
    p = force_state(float(a[0]), p, cos, conf)
    for a0, a1 in zip(a[:-1], a[1:]):
        p = integrate(a0, a1, p, cos, conf)
    o = _order(conf, pmid)
    slab = SlabPM(conf, LocalComm(P))
    states = slab.nbody(slab.distribute(pmid, disp.clone(), vel.clone()), cos, a)
    spmid, sdisp, svel, _ = slab.collect(states)
    assert torch.equal(spmid, pmid[o])
    assert rel_err(sdisp.cpu().numpy(), p.disp[o].cpu().numpy()) < 1e-5
    assert rel_err(svel.cpu().numpy(), p.vel[o].cpu().numpy()) < 1e-5
    # every particle sits in its rank's slab after the routing
    for r, st in enumerate(states):
        cx, _ = slab.cell_x(st.pmid, st.disp)
        assert bool(((cx // slab.nxl) == r).all())


def test_slab_routing_fails_closed_over_capacity():
    from pmpp_b200.slab import LocalComm, SlabPM
    pb, conf, pmid, disp = _setup()
    slab = SlabPM(conf, LocalComm(2), capacity=pmid.shape[0] // 4)
    states = slab.distribute(pmid, disp)
    before = [s.disp.clone() for s in states]
    with pytest.raises(RuntimeError, match="capacity"):
        slab.migrate(states)
    for s, b in zip(states, before):
        assert torch.equal(s.disp, b)


@pytest.mark.parametrize("P", [2, 4])
def test_slab_force_vjp_matches_single_gpu(P):
    from pmpp_b200.gravity import force, force_vjp
    from pmpp_b200.slab import LocalComm, SlabPM
    pb, conf, pmid, disp = _setup(seed=5)
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    ac = torch.from_numpy(np.random.default_rng(7).normal(size=disp.shape).astype(np.float32)).cuda()
    acc, F = force(pmid, disp.clone(), conf, cos.Omega_m)
    dc = torch.zeros_like(disp)
    force_vjp(pmid, disp, conf, cos.Omega_m, F, ac, dc)
    o = _order(conf, pmid)
    slab = SlabPM(conf, LocalComm(P))
    states = slab.distribute(pmid, disp)
    own = slab.owner(pmid, disp)
    acs = [ac[own == r].contiguous() for r in range(P)]
    dcs = slab.force_vjp(states, acs, cos.Omega_m)
    for st, d in zip(states, dcs):
        st.disp_cot = d
    ids = lambda p: (p[:, 0].long() * conf.mesh_shape[1] + p[:, 1].long()) * conf.mesh_shape[2] + p[:, 2].long()
    spmid = torch.cat([s.pmid for s in states])
    sdc = torch.cat([s.disp_cot for s in states])[torch.argsort(ids(spmid))]
    assert rel_err(sdc.cpu().numpy(), dc[o].cpu().numpy()) < 1e-5


@pytest.mark.parametrize("P", [2, 4])
def test_slab_reverse_sweep_matches_single_gpu(P):
    from pmpp_b200.nbody import force_adj, force_state, integrate, integrate_adj
    from pmpp_b200.slab import LocalComm, SlabPM
    a = np.linspace(0.1, 0.5, 4)
    pb, conf, pmid, disp = _setup(spread=1.0, a_custom=a, seed=8)
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    rng = np.random.default_rng(9)
    vel = torch.from_numpy(rng.normal(0, 3.0, disp.shape).astype(np.float32)).cuda()
    dcot = torch.from_numpy(rng.normal(size=disp.shape).astype(np.float32)).cuda()
    vcot = torch.from_numpy(rng.normal(size=disp.shape).astype(np.float32)).cuda()
    # single GPU: forward, then the per-operation reverse sweep
    p = force_state(float(a[0]), pb.Particles(conf, pmid, disp.clone(), vel.clone()), cos, conf)
    for a0, a1 in zip(a[:-1], a[1:]):
        p = integrate(a0, a1, p, cos, conf)
    final_ids = p.pmid
    c = pb.Particles(conf, p.pmid, dcot.clone(), vcot.clone(), torch.zeros_like(dcot))
    om = 0.0
    for a0, a1 in list(zip(a[:-1], a[1:]))[::-1]:
        p, c, om, _ = integrate_adj(a0, a1, p, c, cos, om, conf)
    p, c, om0, _ = force_adj(float(a[0]), p, c, cos, conf)
    om += om0
    o = _order(conf, pmid)
    # slabs: forward, hand the final cotangents to the owners, reverse sweep
    slab = SlabPM(conf, LocalComm(P))
    states = slab.nbody(slab.distribute(pmid, disp.clone(), vel.clone()), cos, a)
    ids = lambda q: (q[:, 0].long() * conf.mesh_shape[1] + q[:, 1].long()) * conf.mesh_shape[2] + q[:, 2].long()
    lookup = torch.empty(int(ids(final_ids).max()) + 1, dtype=torch.long, device="cuda")
    lookup[ids(final_ids)] = torch.arange(final_ids.shape[0], device="cuda")
    for st in states:
        k = lookup[ids(st.pmid)]
        st.disp_cot, st.vel_cot = dcot[k].contiguous(), vcot[k].contiguous()
    states, om_s = slab.nbody_adj(states, cos, a)
    spmid = torch.cat([s.pmid for s in states])
    so = torch.argsort(ids(spmid))
    for name, ref in (("disp", p.disp), ("disp_cot", c.disp), ("vel_cot", c.vel)):
        got = torch.cat([getattr(s, name) for s in states])[so]
        assert rel_err(got.cpu().numpy(), ref[o].cpu().numpy()) < 1e-5, name
    np.testing.assert_allclose(om_s, om, rtol=1e-3)
