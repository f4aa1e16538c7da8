"""GPU parity at the sizes the benchmarks run.

C1 -- 256^3 particles on a 512^3 mesh (4 Mpc/h spacing), position set U
(uniform in the box, PCG64 seed 1) and set K (the 64^3 / 128^3 run's final
positions tiled 4^3, clustered), unit-mean masses:
  * the cell sort bit-exact against the oracle's integer binning (every
    record's uint32 key equals the oracle key of its particle, rows ascending);
  * the density deposit bit-exact against the fixed-point restatement and
    within 1e-6 of the float64 oracle;
  * the 3-channel gather and the scatter / gather adjoint position terms
    within 1e-6, the adjoint deposit within 1e-6;
  * the PM force and its adjoint through the FFT pass chain within 1e-5 of the
    float64 oracle (relative to the field maximum).

C2 -- 512^3 particles on a 1024^3 mesh (2 Mpc/h spacing), the 2LPT state at
a = 0.1 of noise seed 1 (cell keys up to 2^30 - 1):
  * the force through the FFT pass chain within 1e-5 of the independent
    float64 path (pmb_force64: float64 deposit, cuFFT D2Z/Z2D, float64 gather);
  * the force adjoint through the pass chain within 1e-5 of the cuFFT route,
    and the presorted adjoint (sorted records of the last force reused)
    bitwise equal to the sorting one;
  * the kicks folded into the gather bitwise equal to separate updates;
  * the uint32 cell keys of a sample of 4M particles bit-exact against the
    oracle; the deposit on an 8-row x slab bit-exact against the fixed-point
    restatement of the particles that reach it.
The oracle runs threaded over the host cores (a few minutes in all).
"""
import numpy as np
import pytest
import torch

from oracle import pm as opm
from tests.helpers import fixed_point_scatter, rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _threads():
    import os
    opm.set_fft_workers(os.cpu_count() or 1)
    yield
    opm.set_fft_workers(1)
    from pmpp_b200 import runtime
    runtime.release_workspaces()
    torch.cuda.empty_cache()


def _sorted_records(sp):
    """(keys uint32 (n,), perm uint32 (n,)) of a SortedParticles buffer."""
    n = sp.n
    b = sp.buf
    rec = b[:16 * n].view(torch.int32).view(n, 4)
    keys = rec[:, 3].cpu().numpy().view(np.uint32)
    off = (16 * n + 255) // 256 * 256
    perm = b[off:off + 4 * n].view(torch.int32).cpu().numpy().view(np.uint32)
    return keys, perm


def _oracle_keys(pmid, disp, co):
    cell, _, _ = opm.enmesh(pmid, disp, co)
    M = co.mesh_shape
    return ((cell[:, 0] * M[1] + cell[:, 1]) * M[2] + cell[:, 2]).astype(np.uint64)


@pytest.mark.parametrize("which", ["U", "K"])
def test_c1_cic_sort_force_and_adjoints(which):
    import pmpp_b200 as pb
    from pmpp_b200 import microbench as mb
    from pmpp_b200.cic import SortedParticles
    conf = pb.Configuration(4.0, (256, 256, 256), 2, a_start=0.1, device="cuda")
    co = opm.Conf(4.0, (256, 256, 256), mesh_shape=2, a_start=0.1)
    ptcl = mb.uniform_positions(conf) if which == "U" else mb.clustered_positions(conf)
    pmid, disp = ptcl.pmid.cpu().numpy(), ptcl.disp.cpu().numpy()
    n = len(pmid)
    # cell sort
    sp = SortedParticles(ptcl.pmid, ptcl.disp, conf)
    keys, perm = _sorted_records(sp)
    ok = _oracle_keys(pmid, disp, co)
    assert np.array_equal(keys.astype(np.uint64), ok[perm])
    rows = keys // np.uint32(co.mesh_shape[2])
    assert np.all(np.diff(rows.astype(np.int64)) >= 0)
    assert np.array_equal(np.sort(perm), np.arange(n, dtype=np.uint32))
    # density deposit
    rho = pb.scatter(ptcl, conf).cpu().numpy()
    vc = np.float32(conf.mesh_size / conf.ptcl_num)
    exact = fixed_point_scatter(pmid, disp, co, np.full(n, vc, np.float32))
    assert np.array_equal(rho.view(np.uint32), exact.view(np.uint32))
    assert rel_err(rho, opm.scatter(pmid, disp, co)) < 1e-6
    # gather and adjoints
    g = torch.Generator().manual_seed(2)
    mesh3 = torch.randn((3, ) + co.mesh_shape, generator=g)
    cot = torch.randn((n, 3), generator=g)
    m3 = mesh3.numpy().astype(np.float64)
    got = pb.gather(ptcl, conf, mesh3.permute(1, 2, 3, 0).cuda()).cpu().numpy()
    assert rel_err(got, opm.gather(pmid, disp, co, m3)) < 1e-6
    dcs, _ = pb.cic.scatter_vjp(ptcl, conf, mesh3[0].cuda())
    rdcs, _ = opm.scatter_vjp(pmid, disp, co, m3[0])
    assert rel_err(dcs.cpu().numpy(), rdcs) < 1e-6
    dcg, mc = pb.cic.gather_vjp(ptcl, conf, mesh3.permute(1, 2, 3, 0).cuda(), cot.cuda())
    rdcg, rmc = opm.gather_vjp(pmid, disp, co, m3, cot.numpy())
    assert rel_err(dcg.cpu().numpy(), rdcg) < 1e-6
    assert rel_err(np.moveaxis(mc.cpu().numpy(), -1, 0), rmc) < 1e-6
    del mesh3, m3, got, dcs, rdcs, dcg, rdcg, mc, rmc
    # PM force and adjoint through the FFT pass chain
    from pmpp_b200 import _lib
    assert _lib.pmfft_active(*conf.mesh_shape)
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    acc = pb.gravity(1.0, ptcl, cos, conf).cpu().numpy()
    assert rel_err(acc, opm.gravity(pmid, disp, co, 0.3)) < 1e-5
    dc, om = pb.gravity_vjp(1.0, ptcl, cos, conf, cot.cuda())
    rdc, rom = opm.gravity_vjp(pmid, disp, co, 0.3, cot.numpy())
    assert rel_err(dc.cpu().numpy(), rdc) < 1e-5
    np.testing.assert_allclose(om, rom, rtol=1e-5)


def test_c2_force_adjoint_kicks_keys_and_slab():
    import pmpp_b200 as pb
    from pmpp_b200 import _lib, lpt, modes, x64
    from pmpp_b200.gravity import force, force_vjp
    from pmpp_b200.cic import SortedParticles
    n1 = 512
    conf = pb.Configuration(2.0, (n1, ) * 3, 2, a_start=0.1, device="cuda")
    co = opm.Conf(2.0, (n1, ) * 3, mesh_shape=2, a_start=0.1)
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    ptcl = lpt.lpt_full(modes.linear_modes(modes.white_noise_nested(1, conf), cos, conf), cos, conf).ptcl
    pmid, disp = ptcl.pmid, ptcl.disp.clone()
    n = conf.ptcl_num
    om = cos.Omega_m
    assert _lib.pmfft_active(*conf.mesh_shape)
    # force: pass chain (float32) against the float64 path
    acc, F = force(pmid, disp.clone(), conf, om)
    acc = acc.cpu().numpy()
    del F
    from pmpp_b200 import runtime
    runtime.release_workspaces()
    torch.cuda.empty_cache()
    conf64 = pb.Configuration(2.0, (n1, ) * 3, 2, a_start=0.1, device="cuda", float_dtype="float64")
    acc64, F64 = x64.force(pmid, disp.double(), conf64, om)
    acc64 = acc64.cpu().numpy()
    del F64
    runtime.release_workspaces()
    torch.cuda.empty_cache()
    assert rel_err(acc, acc64) < 1e-5
    del acc64
    # adjoint: pass chain against the cuFFT route; presorted bitwise equal
    cot = torch.randn((n, 3), generator=torch.Generator().manual_seed(3)).cuda()
    res = {}
    for route in (True, False):
        _lib.set_pmfft(route)
        try:
            a_, F = force(pmid, disp.clone(), conf, om)
            res[route] = force_vjp(pmid, disp, conf, om, F, cot).cpu().numpy()
            if route:
                d2 = force_vjp(pmid, disp, conf, om, F, cot, presorted=True).cpu().numpy()
                assert np.array_equal(d2.view(np.uint32), res[route].view(np.uint32))
            del a_, F
            runtime.release_workspaces()
            torch.cuda.empty_cache()
        finally:
            _lib.set_pmfft(True)
    assert rel_err(res[True], res[False]) < 1e-5
    del res, d2
    # folded kicks: vel + acc k1 + acc k2, each with two roundings
    vel0 = torch.randn((n, 3), generator=torch.Generator().manual_seed(4)).cuda()
    vel = vel0.clone()
    k1, k2 = 0.37, 0.29
    acc_k, F = force(pmid, disp.clone(), conf, om, vel_kick=vel, kick=k1, kick2=k2)
    del F
    ref = (vel0 + acc_k * np.float32(k1)) + acc_k * np.float32(k2)
    assert torch.equal(vel, ref)
    del vel, vel0, ref, acc_k
    runtime.release_workspaces()
    torch.cuda.empty_cache()
    # uint32 keys near 2^30: a sample against the oracle's binning
    sp = SortedParticles(pmid, disp, conf)
    keys, perm = _sorted_records(sp)
    assert int(keys.max()) < 2**30 and int(keys.max()) > 2**29
    rng = np.random.default_rng(5)
    pick = rng.choice(n, size=4_000_000, replace=False)
    pm_np, dp_np = pmid.cpu().numpy(), disp.cpu().numpy()
    assert np.array_equal(keys[pick].astype(np.uint64), _oracle_keys(pm_np[perm[pick]], dp_np[perm[pick]], co))
    # deposit on the x slab [x0 + 1, x0 + 8]: exactly the particles whose lower
    # corner row lies in [x0, x0 + 8]
    rho = pb.scatter(pb.Particles(conf, pmid, disp), conf)
    x0 = 300
    slab = rho[x0 + 1:x0 + 9].cpu().numpy()
    del rho, sp
    xs = keys // np.uint32(co.mesh_shape[1] * co.mesh_shape[2])
    idx = perm[(xs >= x0) & (xs <= x0 + 8)]
    # restated on a 16-row periodic mesh with the anchors moved down by x0 (the
    # selected corners span rows x0 .. x0 + 9, so nothing wraps)
    pm_s = pm_np[idx].astype(np.int64)
    pm_s[:, 0] -= x0
    vc = np.float32(conf.mesh_size / conf.ptcl_num)
    exact = fixed_point_scatter(pm_s, dp_np[idx], co, np.full(len(idx), vc, np.float32), n_total=n,
                                mesh_shape=(16, co.mesh_shape[1], co.mesh_shape[2]))
    assert np.array_equal(slab.view(np.uint32), exact[1:9].view(np.uint32))
