"""GPU parity of the reference's CIC options: unused slots (Particles.unused_index,
cic/scatter.py:258-272, cic/gather.py:356-357, cic/pallas.py:133-141), a mesh
offset (cic/enmesh.py:128-147, cic/pallas.py:225-238) and an explicit cell size
(cic/enmesh.py:108-127, cic/pallas.py:192-222).

Bars: deposits bit-exact against the fixed-point restatement (tests/helpers.py)
and within 1e-6 of the oracle's float64 sums; gathers and adjoint position
terms within 1e-6 (relative to the field maximum); every output of an unused
slot exactly zero."""
import numpy as np
import pytest
import torch

from oracle import pm as opm
from tests.helpers import fixed_point_scatter, random_particles, rel_err

pytestmark = pytest.mark.gpu


def _setup(shape=(16, 16, 16), mesh=2, seed=0, frac_unused=0.3, tail=True):
    import pmpp_b200 as pb
    conf_o = opm.Conf(2.0, shape, mesh_shape=mesh)
    conf = pb.Configuration(2.0, shape, mesh, device="cuda")
    pmid, disp = random_particles(conf_o, seed, 3.0)
    rng = np.random.default_rng(seed + 11)
    unused = rng.random(len(pmid)) < frac_unused
    if tail:
        unused[-300:] = True  # the last particle tiles entirely unused
    ptcl = pb.Particles(conf, torch.from_numpy(pmid).cuda(), torch.from_numpy(disp).cuda(),
                        unused_index=torch.from_numpy(unused).cuda())
    return pb, conf_o, conf, pmid, disp, ~unused, ptcl


def test_masked_scatter_bit_exact_and_vs_oracle():
    pb, co, conf, pmid, disp, valid, ptcl = _setup()
    got = pb.scatter(ptcl, conf).cpu().numpy()
    vc = np.float32(conf.mesh_size / conf.ptcl_num)
    exact = fixed_point_scatter(pmid, disp, co, np.full(len(pmid), vc, np.float32), valid=valid)
    assert np.array_equal(got.view(np.uint32), exact.view(np.uint32))
    ref = opm.scatter(pmid, disp, co, valid=valid)
    assert rel_err(got, ref) < 1e-6
    # the unused slots carry no mass
    np.testing.assert_allclose(got.sum(), vc * valid.sum(), rtol=1e-5)


def test_masked_scatter_values_ignore_garbage_in_unused_slots():
    pb, co, conf, pmid, disp, valid, ptcl = _setup(seed=1)
    rng = np.random.default_rng(3)
    val = rng.normal(size=(len(pmid), 3)).astype(np.float32)
    val_bad = val.copy()
    val_bad[~valid] = np.nan
    got = pb.scatter(ptcl, conf, val=torch.from_numpy(val_bad).cuda()).cpu().numpy()
    val0 = np.where(valid[:, None], val, 0).astype(np.float32)
    exact = fixed_point_scatter(pmid, disp, co, val0, valid=valid)
    assert np.array_equal(np.moveaxis(got, -1, 0).view(np.uint32), exact.view(np.uint32))


def test_masked_gather_and_kick():
    pb, co, conf, pmid, disp, valid, ptcl = _setup(seed=2)
    rng = np.random.default_rng(7)
    mesh_v = rng.normal(size=co.mesh_shape + (3, )).astype(np.float32)
    got = pb.gather(ptcl, conf, torch.from_numpy(mesh_v).cuda()).cpu().numpy()
    ref = opm.gather(pmid, disp, co, np.moveaxis(mesh_v, -1, 0).astype(np.float64), valid=valid)
    assert rel_err(got, ref) < 1e-6
    assert np.all(got[~valid] == 0)
    # the fused kick leaves the unused slots' velocities untouched
    from pmpp_b200.cic import SortedParticles
    sp = SortedParticles(ptcl.pmid, ptcl.disp, conf, valid=ptcl.valid_mask())
    vel0 = rng.normal(size=(len(pmid), 3)).astype(np.float32)
    vel = torch.from_numpy(vel0).cuda()
    mp = torch.from_numpy(np.ascontiguousarray(np.moveaxis(mesh_v, -1, 0))).cuda()
    acc = sp.gather(mp, vel=vel, kick=0.5).cpu().numpy()
    v = vel.cpu().numpy()
    assert np.array_equal(v[~valid], vel0[~valid])
    np.testing.assert_array_equal(v[valid], (vel0[valid] + acc[valid] * np.float32(0.5)).astype(np.float32))


@pytest.mark.parametrize("staging", [0, 2])
def test_masked_adjoints(staging):
    from pmpp_b200._lib import call
    pb, co, conf, pmid, disp, valid, ptcl = _setup(seed=4)
    rng = np.random.default_rng(9)
    mesh_cot = rng.normal(size=co.mesh_shape).astype(np.float32)
    mesh3 = rng.normal(size=co.mesh_shape + (3, )).astype(np.float32)
    cot = rng.normal(size=(len(pmid), 3)).astype(np.float32)
    call("pmb_set_gather_staging", staging)
    try:
        dc, vcot = pb.cic.scatter_vjp(ptcl, conf, torch.from_numpy(mesh_cot).cuda())
        dg, mc = pb.cic.gather_vjp(ptcl, conf, torch.from_numpy(mesh3).cuda(), torch.from_numpy(cot).cuda())
        g = pb.gather(ptcl, conf, torch.from_numpy(mesh3).cuda()).cpu().numpy()
    finally:
        call("pmb_set_gather_staging", 0)
    rdc, rvc = opm.scatter_vjp(pmid, disp, co, mesh_cot.astype(np.float64), valid=valid)
    assert rel_err(dc.cpu().numpy(), rdc) < 1e-6
    np.testing.assert_allclose(float(vcot), rvc, rtol=1e-5)
    rdg, rmc = opm.gather_vjp(pmid, disp, co, np.moveaxis(mesh3, -1, 0).astype(np.float64), cot, valid=valid)
    assert rel_err(dg.cpu().numpy(), rdg) < 1e-6
    assert rel_err(np.moveaxis(mc.cpu().numpy(), -1, 0), rmc) < 1e-6
    assert np.all(dc.cpu().numpy()[~valid] == 0) and np.all(dg.cpu().numpy()[~valid] == 0)
    assert np.all(g[~valid] == 0)


@pytest.mark.parametrize("offset", [0.5 * 1.0, [0.3, -1.7, 2.25]])
def test_offset_scatter_gather_vjp(offset):
    pb, co, conf, pmid, disp, valid, ptcl = _setup(seed=5, frac_unused=0.0, tail=False)
    ptcl = pb.Particles(conf, ptcl.pmid, ptcl.disp)
    off = np.asarray(offset, dtype=np.float64) * co.cell_size
    got = pb.scatter(ptcl, conf, offset=torch.tensor(off)).cpu().numpy()
    vc = np.float32(conf.mesh_size / conf.ptcl_num)
    exact = fixed_point_scatter(pmid, disp, co, np.full(len(pmid), vc, np.float32), offset=off)
    assert np.array_equal(got.view(np.uint32), exact.view(np.uint32))
    assert rel_err(got, opm.scatter(pmid, disp, co, offset=off)) < 1e-6
    rng = np.random.default_rng(1)
    mesh_v = rng.normal(size=co.mesh_shape).astype(np.float32)
    g = pb.gather(ptcl, conf, torch.from_numpy(mesh_v).cuda(), offset=torch.tensor(off)).cpu().numpy()
    assert rel_err(g, opm.gather(pmid, disp, co, mesh_v.astype(np.float64), offset=off)) < 1e-6
    dc, _ = pb.cic.scatter_vjp(ptcl, conf, torch.from_numpy(mesh_v).cuda(), offset=torch.tensor(off))
    rdc, _ = opm.scatter_vjp(pmid, disp, co, mesh_v.astype(np.float64), offset=off)
    assert rel_err(dc.cpu().numpy(), rdc) < 1e-6
    # a whole-cell offset is a pure index shift of the unshifted deposit
    base = pb.scatter(ptcl, conf).cpu().numpy()
    shifted = pb.scatter(ptcl, conf, offset=co.cell_size).cpu().numpy()
    assert np.array_equal(shifted, np.roll(base, (-1, -1, -1), axis=(0, 1, 2)))


@pytest.mark.parametrize("ratio,shape", [(2.0, (16, 16, 16)), (1.5, (24, 24, 24)), (0.75, (40, 40, 40))])
def test_explicit_cell_size(ratio, shape):
    pb, co, conf, pmid, disp, valid, ptcl = _setup(seed=6, frac_unused=0.2, tail=False)
    cell2 = ratio * co.cell_size
    off = np.array([0.25, 0.0, -0.5]) * co.cell_size
    mesh0 = torch.zeros(shape, device="cuda")
    got = pb.scatter(ptcl, conf, mesh=mesh0, offset=torch.tensor(off), cell_size=cell2).cpu().numpy()
    vc = np.float32(conf.mesh_size / conf.ptcl_num)
    exact = fixed_point_scatter(pmid, disp, co, np.full(len(pmid), vc, np.float32), offset=off, valid=valid,
                                cell_size=cell2, mesh_shape=shape)
    assert np.array_equal(got.view(np.uint32), exact.view(np.uint32))
    ref = opm.scatter(pmid, disp, co, mesh_shape=shape, offset=off, cell_size=cell2, valid=valid)
    assert rel_err(got, ref) < 1e-6
    rng = np.random.default_rng(2)
    mesh_v = rng.normal(size=shape + (2, )).astype(np.float32)
    g = pb.gather(ptcl, conf, torch.from_numpy(mesh_v).cuda(), offset=torch.tensor(off), cell_size=cell2)
    rg = opm.gather(pmid, disp, co, np.moveaxis(mesh_v, -1, 0).astype(np.float64), offset=off, cell_size=cell2,
                    valid=valid)
    assert rel_err(g.cpu().numpy(), rg) < 1e-6
    cot = rng.normal(size=(len(pmid), 2)).astype(np.float32)
    dg, mc = pb.cic.gather_vjp(ptcl, conf, torch.from_numpy(mesh_v).cuda(), torch.from_numpy(cot).cuda(),
                               offset=torch.tensor(off), cell_size=cell2)
    rdg, rmc = opm.gather_vjp(pmid, disp, co, np.moveaxis(mesh_v, -1, 0).astype(np.float64), cot, offset=off,
                              cell_size=cell2, valid=valid)
    assert rel_err(dg.cpu().numpy(), rdg) < 1e-6
    assert rel_err(np.moveaxis(mc.cpu().numpy(), -1, 0), rmc) < 1e-6


def test_explicit_cell_size_equal_to_particle_cell_matches_sorted_path():
    """cell_size == conf.cell_size through the per-particle path agrees with the
    sorted default path within 5e-6: the explicit path forms positions
    pmid * cell + disp in float, the default one bins disp / cell from the
    anchor, so the weights round differently (both exact sums of their own)."""
    pb, co, conf, pmid, disp, valid, ptcl = _setup(seed=8, frac_unused=0.0, tail=False)
    ptcl = pb.Particles(conf, ptcl.pmid, ptcl.disp)
    a = pb.scatter(ptcl, conf).cpu().numpy()
    b = pb.scatter(ptcl, conf, cell_size=co.cell_size).cpu().numpy()
    assert rel_err(b, a) < 5e-6
