"""GPU parity of the cell sort and the CIC kernels against the CPU oracle.

Bars: integer binning and the stable cell order bit-exact; scatter/gather and
their adjoints within 2e-6 of the oracle's float64 accumulation (relative to
the field maximum); scatter results bit-identical across runs and across
particle orderings (fixed-point accumulation).
"""
import ctypes

import numpy as np
import pytest
import torch

from oracle import pm as opm
from tests.helpers import random_particles, rel_err

pytestmark = pytest.mark.gpu

CASES = [((8, 8, 8), 2), ((16, 12, 10), 2), ((9, 9, 9), 1), ((6, 6, 6), 3)]


def _setup(shape, mesh, seed=0, spread=3.0, lattice=True):
    import pmpp_b200 as pb
    conf_o = opm.Conf(2.0, shape, mesh_shape=mesh)
    conf = pb.Configuration(2.0, shape, mesh, device="cuda")
    pmid, disp = random_particles(conf_o, seed, spread, lattice)
    ptcl = pb.Particles(conf, torch.from_numpy(pmid).cuda(), torch.from_numpy(disp).cuda())
    return pb, conf_o, conf, pmid, disp, ptcl


@pytest.mark.parametrize("shape,mesh", CASES)
def test_scatter_density(shape, mesh):
    pb, co, conf, pmid, disp, ptcl = _setup(shape, mesh)
    got = pb.scatter(ptcl, conf).cpu().numpy()
    ref = opm.scatter(pmid, disp, co)
    assert rel_err(got, ref) < 2e-6
    np.testing.assert_allclose(got.sum(), conf.mesh_size, rtol=1e-5)


def test_scatter_deterministic_and_order_independent():
    pb, co, conf, pmid, disp, ptcl = _setup((16, 16, 16), 2, spread=6.0)
    a = pb.scatter(ptcl, conf).cpu().numpy()
    b = pb.scatter(ptcl, conf).cpu().numpy()
    perm = torch.randperm(len(ptcl), generator=torch.Generator().manual_seed(3)).cuda()
    p2 = pb.Particles(conf, ptcl.pmid[perm].contiguous(), ptcl.disp[perm].contiguous())
    c = pb.scatter(p2, conf).cpu().numpy()
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert np.array_equal(a.view(np.uint32), c.view(np.uint32))


def test_scatter_clustered_single_cell():
    pb, co, conf, pmid, disp, ptcl = _setup((8, 8, 8), 2)
    pmid[:] = 3
    disp[:] = 0.25 * co.cell_size
    p = pb.Particles(conf, torch.from_numpy(pmid).cuda(), torch.from_numpy(disp).cuda())
    got = pb.scatter(p, conf).cpu().numpy()
    ref = opm.scatter(pmid, disp, co)
    assert rel_err(got, ref) < 2e-6


@pytest.mark.parametrize("shape,mesh", CASES[:2])
def test_scatter_values_multichannel(shape, mesh):
    pb, co, conf, pmid, disp, ptcl = _setup(shape, mesh, seed=1)
    rng = np.random.default_rng(5)
    val = rng.normal(size=(len(pmid), 3)).astype(np.float32)
    got = pb.scatter(ptcl, conf, val=torch.from_numpy(val).cuda()).cpu().numpy()
    ref = opm.scatter(pmid, disp, co, val=val)
    assert rel_err(np.moveaxis(got, -1, 0), ref) < 2e-6


@pytest.mark.parametrize("shape,mesh", CASES)
def test_gather(shape, mesh):
    pb, co, conf, pmid, disp, ptcl = _setup(shape, mesh, seed=2)
    rng = np.random.default_rng(7)
    mesh_v = rng.normal(size=co.mesh_shape + (3, )).astype(np.float32)
    got = pb.gather(ptcl, conf, torch.from_numpy(mesh_v).cuda()).cpu().numpy()
    ref = opm.gather(pmid, disp, co, np.moveaxis(mesh_v, -1, 0).astype(np.float64))
    assert rel_err(got, ref) < 2e-6


@pytest.mark.parametrize("shape,mesh", CASES[:2])
def test_scatter_vjp(shape, mesh):
    pb, co, conf, pmid, disp, ptcl = _setup(shape, mesh, seed=3)
    rng = np.random.default_rng(8)
    mc = rng.normal(size=co.mesh_shape).astype(np.float32)
    dc, vc = pb.scatter_vjp(ptcl, conf, torch.from_numpy(mc).cuda())
    rdc, rvc = opm.scatter_vjp(pmid, disp, co, mc.astype(np.float64))
    assert rel_err(dc.cpu().numpy(), rdc) < 5e-6
    np.testing.assert_allclose(float(vc), rvc, rtol=1e-5)


@pytest.mark.parametrize("shape,mesh", CASES[:2])
def test_gather_vjp(shape, mesh):
    pb, co, conf, pmid, disp, ptcl = _setup(shape, mesh, seed=4)
    rng = np.random.default_rng(9)
    mesh_v = rng.normal(size=co.mesh_shape + (3, )).astype(np.float32)
    vcot = rng.normal(size=(len(pmid), 3)).astype(np.float32)
    dc, mc = pb.gather_vjp(ptcl, conf, torch.from_numpy(mesh_v).cuda(), torch.from_numpy(vcot).cuda())
    rdc, rmc = opm.gather_vjp(pmid, disp, co, np.moveaxis(mesh_v, -1, 0).astype(np.float64), vcot)
    assert rel_err(dc.cpu().numpy(), rdc) < 5e-6
    assert rel_err(np.moveaxis(mc.cpu().numpy(), -1, 0), rmc) < 2e-6


@pytest.mark.parametrize("shape,mesh", CASES)
def test_sort_by_cell_bit_exact(shape, mesh):
    pb, co, conf, pmid, disp, ptcl = _setup(shape, mesh, seed=5, spread=5.0)
    from pmpp_b200 import sort as pbsort
    keys, perm = pbsort.sort_by_cell(ptcl, conf)
    rk, rp = opm.sort_by_cell(pmid, disp, co)
    assert np.array_equal(keys.cpu().numpy().astype(np.int64), rk[rp])
    assert np.array_equal(perm.cpu().numpy().astype(np.int64), rp)


def test_row_bins_match_reference_binning():
    """The row of every sorted record equals the reference enmesh lower corner."""
    pb, co, conf, pmid, disp, ptcl = _setup((16, 12, 10), 2, seed=6, spread=8.0)
    from pmpp_b200.cic import SortedParticles
    sp = SortedParticles(ptcl.pmid, ptcl.disp, conf)
    n = len(pmid)
    raw = sp.buf[:16 * n].view(torch.int32).reshape(n, 4).cpu().numpy()
    off = ((16 * n + 255) // 256) * 256
    perm = sp.buf[off:off + 4 * n].view(torch.int32).cpu().numpy().astype(np.int64)
    keys = raw[:, 3].astype(np.uint32).astype(np.int64)
    ref = opm.cell_key(pmid, disp, co)
    assert np.array_equal(keys, ref[perm])
    assert np.array_equal(np.sort(perm), np.arange(n))
    rows = keys // co.mesh_shape[2]
    assert np.all(np.diff(rows) >= 0)


def _exact_case(concentrate, seed=5):
    """2^17 particles on an 8^3 mesh; with concentrate, 100000 of them in one
    mesh row, so the scatter blocks next to it hold more than 2^16 particles
    (64-bit accumulation) and the others fewer (split 32-bit accumulation)."""
    import pmpp_b200 as pb
    co = opm.Conf(2.0, (8, 8, 8), mesh_shape=1)
    conf = pb.Configuration(2.0, (8, 8, 8), 1, device="cuda")
    rng = np.random.default_rng(seed)
    n = 1 << 17
    pmid = rng.integers(0, 8, size=(n, 3)).astype(np.int16)
    disp = rng.uniform(-3.0, 3.0, size=(n, 3)).astype(np.float32)
    if concentrate:
        pmid[:100000, 0] = 3
        pmid[:100000, 1] = 3
        disp[:100000, :2] = rng.uniform(0.0, 1.99, size=(100000, 2)).astype(np.float32)
    return pb, co, conf, pmid, disp


@pytest.mark.parametrize("concentrate", [False, True])
def test_scatter_bit_exact_fixed_point(concentrate):
    from pmpp_b200.cic import SortedParticles
    from tests.helpers import fixed_point_scatter
    pb, co, conf, pmid, disp = _exact_case(concentrate)
    sp = SortedParticles(torch.from_numpy(pmid).cuda(), torch.from_numpy(disp).cuda(), conf)
    got = sp.scatter(val_const=1.75)[0].cpu().numpy()
    ref = fixed_point_scatter(pmid, disp, co, np.full(len(pmid), 1.75, np.float32))
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


@pytest.mark.parametrize("concentrate", [False, True])
def test_scatter_sorted_values_bit_exact(concentrate):
    """3-channel signed values: particle-order and sorted-order inputs give the
    same bits, equal to the fixed-point restatement."""
    from pmpp_b200.cic import SortedParticles
    from tests.helpers import fixed_point_scatter
    pb, co, conf, pmid, disp = _exact_case(concentrate, seed=6)
    rng = np.random.default_rng(7)
    vals = rng.normal(size=(len(pmid), 3)).astype(np.float32)
    sp = SortedParticles(torch.from_numpy(pmid).cuda(), torch.from_numpy(disp).cuda(), conf)
    v = torch.from_numpy(vals).cuda()
    mesh = torch.from_numpy(rng.normal(size=(3, 8, 8, 8)).astype(np.float32)).cuda()
    u_sorted = torch.empty_like(v)
    sp.interp_grad(mesh, u=v, u_sorted=u_sorted)
    a = sp.scatter(val=v, channels=3).cpu().numpy()
    b = sp.scatter(val=u_sorted, channels=3, val_sorted=True).cpu().numpy()
    ref = fixed_point_scatter(pmid, disp, co, vals)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert np.array_equal(a.view(np.uint32), ref.view(np.uint32))


@pytest.mark.parametrize("mode", [1, 2])
@pytest.mark.parametrize("shape,mesh", [((8, 8, 8), 2), ((16, 12, 12), 2), ((32, 32, 32), 1)])
def test_staged_kernels_match_direct_bitwise(shape, mesh, mode):
    """Mesh rows staged in shared memory by bulk copies give the same bits as
    direct loads (a mesh pointer that is not 16-byte aligned takes the direct
    path); no bounded wait gives up."""
    from pmpp_b200 import _lib
    from pmpp_b200.cic import SortedParticles
    _lib.call("pmb_set_gather_staging", mode)
    try:
        _staged_vs_direct(shape, mesh)
    finally:
        _lib.call("pmb_set_gather_staging", 0)


def _staged_vs_direct(shape, mesh):
    from pmpp_b200 import _lib
    from pmpp_b200.cic import SortedParticles
    pb, co, conf, pmid, disp, ptcl = _setup(shape, mesh, spread=4.0)
    sp = SortedParticles(ptcl.pmid, ptcl.disp, conf)
    nx, ny, nz = conf.mesh_shape
    M = nx * ny * nz
    rng = np.random.default_rng(9)
    vals = torch.from_numpy(rng.normal(size=3 * M).astype(np.float32)).cuda()
    big = torch.zeros(3 * M + 4, dtype=torch.float32, device="cuda")
    aligned = big[:3 * M].view(3, nx, ny, nz)
    aligned.view(-1).copy_(vals)
    shifted = big[1:3 * M + 1].view(3, nx, ny, nz)
    u = torch.from_numpy(rng.normal(size=(len(ptcl), 3)).astype(np.float32)).cuda()
    a = sp.gather(aligned).clone()
    da, wa = sp.interp_grad(aligned, u=u, wsum=True)
    da, wa = da.clone(), wa.clone()
    shifted.view(-1).copy_(vals)
    b = sp.gather(shifted)
    db, wb = sp.interp_grad(shifted, u=u, wsum=True)
    assert torch.equal(a, b)
    assert torch.equal(da, db) and torch.equal(wa, wb)
    assert _lib.wait_timeouts() == 0
