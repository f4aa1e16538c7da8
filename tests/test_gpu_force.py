"""GPU parity of the PM force, the KDK integration and the reverse sweep.

Bars (float32 kernels vs the float64-FFT oracle with float32 binning):
force and force adjoint within 1e-5 of the field maximum; a uniform lattice
feels no force (reference test_deep_gravity_spectral.py:253-275: atol 3e-7,
momentum < 2e-5); 3-step N-body states within 1e-4 and the adjoint
cotangents within 1e-3 (chaotic growth of float32 rounding).
"""
import numpy as np
import pytest
import torch

from oracle import cosmology as ocos
from oracle import pm as opm
from tests.helpers import random_particles, rel_err

pytestmark = pytest.mark.gpu


def _confs(shape=(16, 16, 16), mesh=2, spacing=4.0, a_custom=None, **kw):
    import pmpp_b200 as pb
    co = opm.Conf(spacing, shape, mesh_shape=mesh, a_start=0.1, a_custom=a_custom, **kw)
    c = pb.Configuration(spacing, shape, mesh, a_start=0.1, a_custom=a_custom, device="cuda", **kw)
    return pb, co, c


def test_uniform_lattice_zero_force():
    pb, co, conf = _confs()
    ptcl = pb.Particles.gen_grid(conf)
    acc = pb.gravity(1.0, ptcl, pb.boltzmann(pb.SimpleLCDM(conf)), conf)
    assert float(acc.abs().max()) < 3e-7
    assert float(acc.double().sum(0).abs().max()) < 2e-5


@pytest.mark.parametrize("mesh", [1, 2])
def test_gravity_matches_oracle(mesh):
    pb, co, conf = _confs(mesh=mesh)
    pmid, disp = random_particles(co, seed=11, spread=2.0)
    ptcl = pb.Particles(conf, torch.from_numpy(pmid).cuda(), torch.from_numpy(disp).cuda())
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    acc = pb.gravity(1.0, ptcl, cos, conf).cpu().numpy()
    ref = opm.gravity(pmid, disp, co, 0.3)
    assert rel_err(acc, ref) < 1e-5


def test_gravity_vjp_matches_oracle():
    pb, co, conf = _confs()
    pmid, disp = random_particles(co, seed=12, spread=2.0)
    ptcl = pb.Particles(conf, torch.from_numpy(pmid).cuda(), torch.from_numpy(disp).cuda())
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    ac = np.random.default_rng(1).normal(size=disp.shape).astype(np.float32)
    dc, om = pb.gravity_vjp(1.0, ptcl, cos, conf, torch.from_numpy(ac).cuda())
    rdc, rom = opm.gravity_vjp(pmid, disp, co, 0.3, ac)
    assert rel_err(dc.cpu().numpy(), rdc) < 1e-5
    np.testing.assert_allclose(om, rom, rtol=1e-5)


def _nbody_inputs(co, conf, pb, seed=21):
    pmid, disp = random_particles(co, seed=seed, spread=1.0)
    vel = np.random.default_rng(seed + 1).normal(0, 0.5, size=disp.shape).astype(np.float32)
    ptcl = pb.Particles(conf, torch.from_numpy(pmid).cuda(), torch.from_numpy(disp).cuda(),
                        torch.from_numpy(vel).cuda())
    return pmid, disp, vel, ptcl


def test_nbody_forward_matches_oracle():
    a = np.linspace(0.1, 1.0, 4)
    pb, co, conf = _confs(a_custom=a)
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    oc = opm.boltzmann(ocos.Cosmo(), co)
    pmid, disp, vel, ptcl = _nbody_inputs(co, conf, pb)
    out = pb.nbody(ptcl, cos, conf)
    rd, rv, ra = opm.nbody(pmid, disp, vel, co, oc)
    assert rel_err(out.disp.cpu().numpy(), rd) < 1e-4
    assert rel_err(out.vel.cpu().numpy(), rv) < 1e-4
    assert rel_err(out.acc.cpu().numpy(), ra) < 1e-4


def test_nbody_adjoint_matches_oracle():
    a = np.linspace(0.1, 1.0, 3)
    pb, co, conf = _confs(a_custom=a)
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    oc = opm.boltzmann(ocos.Cosmo(), co)
    pmid, disp, vel, ptcl = _nbody_inputs(co, conf, pb, seed=31)
    run = pb.NBodyRun(conf, cos)
    out = run.forward(ptcl)
    rng = np.random.default_rng(4)
    dcot = rng.normal(size=disp.shape).astype(np.float32)
    vcot = rng.normal(size=disp.shape).astype(np.float32)
    cot = pb.Particles(conf, ptcl.pmid, torch.from_numpy(dcot).cuda(), torch.from_numpy(vcot).cuda(),
                       torch.zeros_like(out.disp))
    p0, c0, om = run.adjoint(out, cot)
    rd, rv, ra = opm.nbody(pmid, disp, vel, co, oc)
    _, _, rdc, rvc, rom = opm.nbody_adj(pmid, rd, rv, ra, dcot, vcot, np.zeros_like(dcot), co, oc)
    assert rel_err(c0.disp.cpu().numpy(), rdc) < 1e-3
    assert rel_err(c0.vel.cpu().numpy(), rvc) < 1e-3
    np.testing.assert_allclose(om, rom, rtol=1e-3)
    # the reverse sweep reconstructs the initial state up to float32 round-off
    assert rel_err(p0.disp.cpu().numpy(), disp) < 1e-4


@pytest.mark.parametrize("staged", [False, True])
@pytest.mark.parametrize("shape,mesh", [((16, 16, 16), 2), ((32, 32, 32), 4)])
def test_force_vjp_presorted_matches_sorting_route(staged, shape, mesh):
    """The reverse sweep reuses the force recompute's cell-sorted records."""
    import contextlib

    from pmpp_b200.gravity import force, force_vjp
    from pmpp_b200.runtime import StageTimer
    pb, co, conf = _confs(shape=shape, mesh=mesh)
    pmid, disp = random_particles(co, seed=14, spread=2.0)
    pm, d = torch.from_numpy(pmid).cuda(), torch.from_numpy(disp).cuda()
    ac = torch.from_numpy(np.random.default_rng(3).normal(size=disp.shape).astype(np.float32)).cuda()
    with (StageTimer() if staged else contextlib.nullcontext()):
        _, F = force(pm, d, conf, 0.3)
        got = force_vjp(pm, d, conf, 0.3, F, ac, presorted=True)
        ref = force_vjp(pm, d, conf, 0.3, F, ac)
    assert torch.equal(got, ref)


@pytest.mark.parametrize("two,zero", [(0, 0), (1, 0), (1, 1), (0, 1)])
def test_kick_adj2_matches_separate_kernels(two, zero):
    """The merged kick adjoint applies the same float operations as separate ones."""
    from pmpp_b200._lib import call
    from pmpp_b200.runtime import stream_handle
    g = torch.Generator().manual_seed(8)
    n = 3 * 100003
    vel, acc, vc, ac = (torch.randn(n, generator=g).cuda() for _ in range(4))
    s = stream_handle(vel.device)
    ka, kb = 0.37, -1.21
    v1, c1 = vel.clone(), ac.clone()
    if zero:
        c1.zero_()
    d1 = torch.zeros(3, dtype=torch.float64, device="cuda")
    call("pmb_kick_adj", v1.data_ptr(), acc.data_ptr(), vc.data_ptr(), c1.data_ptr(), n, ka, d1[0:].data_ptr(), s)
    if two:
        call("pmb_kick_adj", v1.data_ptr(), acc.data_ptr(), vc.data_ptr(), c1.data_ptr(), n, kb, d1[1:].data_ptr(), s)
    call("pmb_dot", c1.data_ptr(), acc.data_ptr(), n, d1[2:].data_ptr(), s)
    v2, c2 = vel.clone(), ac.clone()
    d2 = torch.zeros(3, dtype=torch.float64, device="cuda")
    call("pmb_kick_adj2", v2.data_ptr(), acc.data_ptr(), vc.data_ptr(), c2.data_ptr(), n, ka, kb, two, zero,
         d2[0:].data_ptr(), d2[1:].data_ptr(), d2[2:].data_ptr(), s)
    assert torch.equal(v1, v2) and torch.equal(c1, c2)
    torch.testing.assert_close(d1, d2, rtol=1e-12, atol=1e-9)


@pytest.mark.parametrize("two", [0, 1])
def test_kick_adj3_matches_drift_cot_then_kick_adj2(two):
    """The drift cotangent folded into the kick adjoints' pass gives the
    separate pmb_drift_cot_adj + pmb_kick_adj2 results bit for bit (the dots to
    summation-order rounding)."""
    from pmpp_b200._lib import call
    from pmpp_b200.runtime import stream_handle
    g = torch.Generator().manual_seed(9)
    n = 3 * 100003
    vel, acc, vc, ac, dc = (torch.randn(n, generator=g).cuda() for _ in range(5))
    s = stream_handle(vel.device)
    ka, kb, dd = 0.37, -1.21, 0.83
    v1, w1, c1 = vel.clone(), vc.clone(), ac.clone()
    d1 = torch.zeros(4, dtype=torch.float64, device="cuda")
    call("pmb_drift_cot_adj", v1.data_ptr(), dc.data_ptr(), w1.data_ptr(), n, dd, d1[3:].data_ptr(), s)
    call("pmb_kick_adj2", v1.data_ptr(), acc.data_ptr(), w1.data_ptr(), c1.data_ptr(), n, ka, kb, two, 0,
         d1[0:].data_ptr(), d1[1:].data_ptr(), d1[2:].data_ptr(), s)
    v2, w2, c2 = vel.clone(), vc.clone(), ac.clone()
    d2 = torch.zeros(4, dtype=torch.float64, device="cuda")
    call("pmb_kick_adj3", v2.data_ptr(), acc.data_ptr(), w2.data_ptr(), c2.data_ptr(), n, ka, kb, two, 0,
         d2[0:].data_ptr(), d2[1:].data_ptr(), d2[2:].data_ptr(), dc.data_ptr(), dd, d2[3:].data_ptr(), s)
    assert torch.equal(v1, v2) and torch.equal(w1, w2) and torch.equal(c1, c2)
    torch.testing.assert_close(d1, d2, rtol=1e-12, atol=1e-9)


@pytest.mark.parametrize("staged", [False, True])
def test_reverse_sweep_overlap_matches_sequential(staged):
    """The force recompute on a side stream gives the sequential sweep's result."""
    import contextlib

    from pmpp_b200.runtime import StageTimer
    a = np.linspace(0.1, 1.0, 5)
    pb, co, conf = _confs(shape=(32, 32, 32), mesh=4, a_custom=a)
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    pmid, disp, vel, ptcl = _nbody_inputs(co, conf, pb, seed=41)
    rng = np.random.default_rng(5)
    dcot = torch.from_numpy(rng.normal(size=disp.shape).astype(np.float32)).cuda()
    vcot = torch.from_numpy(rng.normal(size=disp.shape).astype(np.float32)).cuda()
    res = {}
    for overlap in (False, True):
        run = pb.NBodyRun(conf, cos, overlap=overlap)
        with (StageTimer() if staged else contextlib.nullcontext()):
            out = run.forward(ptcl)
            cot = pb.Particles(conf, ptcl.pmid, dcot, vcot, torch.zeros_like(out.disp))
            res[overlap] = run.adjoint(out, cot)
    (p0, c0, om0), (p1, c1, om1) = res[False], res[True]
    for x, y in ((p0.disp, p1.disp), (p0.vel, p1.vel), (c0.disp, c1.disp), (c0.vel, c1.vel)):
        assert torch.equal(x, y)
    np.testing.assert_allclose(om1, om0, rtol=1e-9)


_PGD = dict(alpha0=0.3, A=0.4, B=0.1, kl=0.1, ks=1.0)


def _oracle_transfer(model, co, a):
    window = opm.window_gain(co)
    pgd = opm.pgd_transfer(co, a, **_PGD)
    soft = opm.softening_transfer(co, 0.6, 0.5, 1.0)
    return {"pm_window": window, "pgd": pgd, "softening": soft, "windowed_pgd": window * pgd,
            "pm_window+softening": window * soft}.get(model.replace(":interlaced", ""))


@pytest.mark.parametrize("model", ["pm_window", "fastpm_1_4", "fastpm_3_4", "pgd", "softening", "windowed_pgd",
                                   "pm_window+softening", "pm_window:interlaced", "windowed_pgd:interlaced"])
@pytest.mark.parametrize("pmfft", [True, False])
def test_force_with_analytic_corrections_matches_oracle(model, pmfft):
    """The window compensation (corrections/window.py:229-265), the discrete
    Laplacian (gravity.py:122-171), FastPM's 4-point gradient
    (gravity.py:355-391), the PGD transfer at a = 0.5 (corrections/pgd.py:
    154-237), high-k softening (corrections/softening.py:49-80) and their
    products (corrections/combined.py) in the force and its adjoint, through
    the FFT pass chain (128^3 mesh) and the cuFFT route, within 1e-5 of the
    oracle."""
    import pmpp_b200 as pb
    from pmpp_b200 import _lib
    from pmpp_b200.corrections import init_potential_correction
    co = opm.Conf(4.0, (64, 64, 64), mesh_shape=2, a_start=0.1)
    conf = pb.Configuration(4.0, (64, 64, 64), 2, a_start=0.1, device="cuda")
    pmid, disp = random_particles(co, 5, 1.0)
    a = 0.5
    il = model.endswith(":interlaced")
    corr = init_potential_correction(model.replace(":interlaced", ""), strength=0.6, start=0.5, interlacing=il,
                                     **_PGD)
    gk = "discrete_laplacian" if corr.green_kernel == 1 else "continuum"
    kernel = opm.potential_kernel(co, gk, _oracle_transfer(model, co, a))
    grad = corr.gradient_kernel
    ref = opm.gravity(pmid, disp, co, 0.3, kernel=kernel, gradient=grad, interlacing=il)
    rng = np.random.default_rng(6)
    acc_cot = rng.normal(size=disp.shape).astype(np.float32)
    rdc, rom = opm.gravity_vjp(pmid, disp, co, 0.3, acc_cot, kernel=kernel, gradient=grad, interlacing=il)
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    p = pb.Particles(conf, torch.from_numpy(pmid).cuda(), torch.from_numpy(disp).cuda())
    _lib.set_pmfft(pmfft)
    try:
        assert _lib.pmfft_active(*conf.mesh_shape) == pmfft
        acc = pb.gravity(a, p, cos, conf, correction=corr).cpu().numpy()
        dc, om = pb.gravity_vjp(a, p, cos, conf, torch.from_numpy(acc_cot).cuda(), correction=corr)
    finally:
        _lib.set_pmfft(True)
    assert rel_err(acc, ref) < 1e-5
    assert rel_err(dc.cpu().numpy(), rdc) < 1e-5
    np.testing.assert_allclose(om, rom, rtol=1e-5)
    if il:  # interlacing is a different force from the plain one
        plain = opm.gravity(pmid, disp, co, 0.3, kernel=kernel, gradient=grad)
        assert rel_err(acc, plain) > 1e-3


@pytest.mark.parametrize("staged", [False, True])
def test_interlaced_presorted_adjoint_and_lattice(staged):
    """The interlaced force adjoint reusing both sorted record sets equals the
    sorting one bitwise; a uniform lattice feels no interlaced force."""
    import contextlib

    from pmpp_b200.corrections import init_potential_correction
    from pmpp_b200.gravity import force, force_vjp
    from pmpp_b200.runtime import StageTimer
    pb, co, conf = _confs(shape=(32, 32, 32), mesh=2)
    corr = init_potential_correction("pm_window", interlacing=True)
    pmid, disp = random_particles(co, seed=15, spread=2.0)
    pm, d = torch.from_numpy(pmid).cuda(), torch.from_numpy(disp).cuda()
    ac = torch.from_numpy(np.random.default_rng(3).normal(size=disp.shape).astype(np.float32)).cuda()
    with (StageTimer() if staged else contextlib.nullcontext()):
        _, F = force(pm, d, conf, 0.3, a=1.0, correction=corr, lane="1")
        got = force_vjp(pm, d, conf, 0.3, F, ac, a=1.0, correction=corr, presorted=True, sorted_lane="1")
        ref = force_vjp(pm, d, conf, 0.3, F, ac, a=1.0, correction=corr)
    assert torch.equal(got, ref)
    grid = pb.Particles.gen_grid(conf)
    acc = pb.gravity(1.0, grid, pb.boltzmann(pb.SimpleLCDM(conf)), conf, correction=corr)
    assert float(acc.abs().max()) < 3e-7


@pytest.mark.parametrize("il", [False, True])
def test_windowed_nbody_forward_and_adjoint_match_oracle(il):
    """Two KDK steps and the reverse sweep with the window correction, plain
    and interlaced (gravity.py:809-811 inside integrator.py:689-837)."""
    from pmpp_b200.corrections import init_potential_correction
    a = np.linspace(0.1, 1.0, 3)
    pb, co, conf = _confs(a_custom=a)
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    oc = opm.boltzmann(ocos.Cosmo(), co)
    corr = init_potential_correction("pm_window", interlacing=il)
    kern = opm.potential_kernel(co, "discrete_laplacian", opm.window_gain(co))
    pmid, disp, vel, ptcl = _nbody_inputs(co, conf, pb, seed=33)
    run = pb.NBodyRun(conf, cos, corr)
    out = run.forward(ptcl)
    rd, rv, ra = opm.nbody(pmid, disp, vel, co, oc, kern, interlacing=il)
    assert rel_err(out.disp.cpu().numpy(), rd) < 1e-4
    assert rel_err(out.vel.cpu().numpy(), rv) < 1e-4
    assert rel_err(out.acc.cpu().numpy(), ra) < 1e-4
    rng = np.random.default_rng(5)
    dcot = rng.normal(size=disp.shape).astype(np.float32)
    vcot = rng.normal(size=disp.shape).astype(np.float32)
    cot = pb.Particles(conf, ptcl.pmid, torch.from_numpy(dcot).cuda(), torch.from_numpy(vcot).cuda(),
                       torch.zeros_like(out.disp))
    p0, c0, om = run.adjoint(out, cot)
    terms = []
    _, _, rdc, rvc, rom = opm.nbody_adj(pmid, rd, rv, ra, dcot, vcot, np.zeros_like(dcot), co, oc, kern,
                                        interlacing=il, om_terms=terms)
    assert rel_err(c0.disp.cpu().numpy(), rdc) < 1e-3
    assert rel_err(c0.vel.cpu().numpy(), rvc) < 1e-3
    # the Omega_m cotangent is a sum of force and time-factor terms that can
    # cancel to ~1% of their size (-4.97 from terms up to 370 for the
    # interlaced run): its error is bounded against the terms' scale
    assert abs(om - rom) < 1e-4 * sum(abs(t) for t in terms)


def test_pgd_windowed_nbody_forward_and_adjoint_match_oracle():
    """Two KDK steps and the reverse sweep with the window compensation times
    the scale-factor dependent PGD transfer: every force, its adjoint and each
    recomputed force take their positions' scale factor (integrator.py:
    620-686), as the oracle's run and sweep with a kernel per scale factor."""
    from pmpp_b200.corrections import init_potential_correction
    a = np.linspace(0.1, 1.0, 3)
    pb, co, conf = _confs(a_custom=a)
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    oc = opm.boltzmann(ocos.Cosmo(), co)
    corr = init_potential_correction("windowed_pgd", **_PGD)
    kern = lambda s: opm.potential_kernel(co, "discrete_laplacian", opm.window_gain(co) * opm.pgd_transfer(co, s, **_PGD))
    pmid, disp, vel, ptcl = _nbody_inputs(co, conf, pb, seed=35)
    run = pb.NBodyRun(conf, cos, corr)
    out = run.forward(ptcl)
    rd, rv, ra = opm.nbody(pmid, disp, vel, co, oc, kern)
    assert rel_err(out.disp.cpu().numpy(), rd) < 1e-4
    assert rel_err(out.vel.cpu().numpy(), rv) < 1e-4
    assert rel_err(out.acc.cpu().numpy(), ra) < 1e-4
    rng = np.random.default_rng(6)
    dcot = rng.normal(size=disp.shape).astype(np.float32)
    vcot = rng.normal(size=disp.shape).astype(np.float32)
    cot = pb.Particles(conf, ptcl.pmid, torch.from_numpy(dcot).cuda(), torch.from_numpy(vcot).cuda(),
                       torch.zeros_like(out.disp))
    _, c0, om = run.adjoint(out, cot)
    terms = []
    _, _, rdc, rvc, rom = opm.nbody_adj(pmid, rd, rv, ra, dcot, vcot, np.zeros_like(dcot), co, oc, kern,
                                        om_terms=terms)
    assert rel_err(c0.disp.cpu().numpy(), rdc) < 1e-3
    assert rel_err(c0.vel.cpu().numpy(), rvc) < 1e-3
    assert abs(om - rom) < 1e-4 * sum(abs(t) for t in terms)


def test_per_operation_adjoints_match_the_fused_reverse_sweep():
    """kick_adj / drift_adj_from_output / force_adj / integrate_adj
    (integrator.py:429-837) stepped by hand from the final state reproduce the
    fused reverse sweep's cotangents (NBodyRun.adjoint) within 1e-6, and the
    Omega_m cotangent within 1e-6."""
    a = np.linspace(0.1, 1.0, 4)
    pb, co, conf = _confs(a_custom=a)
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    pmid, disp, vel, ptcl = _nbody_inputs(co, conf, pb, seed=41)
    run = pb.NBodyRun(conf, cos)
    out = run.forward(ptcl)
    rng = np.random.default_rng(8)
    dcot = torch.from_numpy(rng.normal(size=disp.shape).astype(np.float32)).cuda()
    vcot = torch.from_numpy(rng.normal(size=disp.shape).astype(np.float32)).cuda()
    cot = pb.Particles(conf, ptcl.pmid, dcot, vcot, torch.zeros_like(dcot))
    p_f, c_f, om_f = run.adjoint(out, cot)
    p, c, om = out, cot, 0.0
    for a_prev, a_next in list(zip(a[:-1], a[1:]))[::-1]:
        p, c, om, _ = pb.integrate_adj(a_prev, a_next, p, c, cos, om, conf)
    p, c, om_i, _ = pb.force_adj(float(a[0]), p, c, cos, conf)
    om += om_i
    assert rel_err(c.disp.cpu().numpy(), c_f.disp.cpu().numpy()) < 1e-6
    assert rel_err(c.vel.cpu().numpy(), c_f.vel.cpu().numpy()) < 1e-6
    np.testing.assert_allclose(om, om_f, rtol=1e-6)
    assert rel_err(p.disp.cpu().numpy(), p_f.disp.cpu().numpy()) < 1e-6
