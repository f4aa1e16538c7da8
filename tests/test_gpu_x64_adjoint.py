"""float64 adjoints (the reference's x64 gradients, tests/test_grad_nbody.py:
118-179 and tests/test_finite_diff.py:87-124) against the float64 oracle.

Bars: one force adjoint within 1e-12 of the oracle's transpose (relative to
the field maximum) and its Omega_m cotangent within 1e-12; a 3-step run of a
strongly perturbed random state (velocities of 0.5, crossing orbits) and its
reverse sweep: final positions and the position / velocity cotangents within
1e-10 (measured 3.5e-11 / 5.1e-11 / 4.3e-11: the orbits amplify float64
rounding, the reconstructed initial state agrees to 1.4e-15), the Omega_m
cotangent within 1e-5 (measured 5.4e-6: the oracle takes the time factors'
Omega_m derivatives by central differences of step 1e-4, the build by
complex step); stepping the per-operation adjoints reproduces the sweep
within 1e-13; a fourth-order finite difference of the float64 run (step
1e-4) matches the sweep's directional derivative within 1e-6, as the
reference's protocol.  The float64 LPT adjoint (tests/test_grad_lpt.py:
82-134) against fourth-order differences of the 2LPT displacements, which
are quadratic in the modes, so the difference is exact up to rounding (1e-9);
the gradient of a density loss through linear modes, 2LPT, a 2-step run and
the deposit w.r.t. the white-noise modes against differences (1e-6)."""
import numpy as np
import pytest
import torch

from oracle import cosmology as ocos
from oracle import pm as opm

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _confs(n=16, mesh=2, a=None, spacing=4.0):
    import pmpp_b200 as pb
    co = opm.Conf(spacing, (n, n, n), mesh_shape=mesh, a_start=0.1, a_custom=a, float_dtype=np.float64)
    conf = pb.Configuration(spacing, (n, n, n), mesh, a_start=0.1, a_custom=a, float_dtype="float64",
                            device="cuda")
    return pb, co, conf


def _state(co, conf, pb, seed, spread=2.0, vel_sd=0.5):
    rng = np.random.default_rng(seed)
    pmid, disp = opm.gen_grid(co)
    disp = disp + rng.normal(0, spread, size=disp.shape)
    vel = rng.normal(0, vel_sd, size=disp.shape)
    ptcl = pb.Particles(conf, torch.from_numpy(pmid).cuda(), torch.from_numpy(disp).cuda(),
                        torch.from_numpy(vel).cuda())
    return pmid, disp, vel, ptcl


@pytest.mark.parametrize("mesh", [1, 2])
def test_force_adjoint_float64(mesh):
    pb, co, conf = _confs(16, mesh)
    pmid, disp, _, ptcl = _state(co, conf, pb, 1)
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    ac = np.random.default_rng(2).normal(size=disp.shape)
    dc, om = pb.gravity_vjp(1.0, ptcl, cos, conf, torch.from_numpy(ac).cuda())
    assert dc.dtype == torch.float64
    rdc, rom = opm.gravity_vjp(pmid, disp, co, cos.Omega_m, ac)
    assert _rel(dc.cpu().numpy(), rdc) < 1e-12
    np.testing.assert_allclose(om, rom, rtol=1e-12)


def test_reverse_sweep_float64_matches_oracle():
    a = np.linspace(0.1, 1.0, 4)
    pb, co, conf = _confs(16, 2, a)
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    oc = opm.boltzmann(ocos.Cosmo(), co)
    pmid, disp, vel, ptcl = _state(co, conf, pb, 3, 1.0)
    run = pb.NBodyRun(conf, cos)
    out = run.forward(ptcl)
    rd, rv, ra = opm.nbody(pmid, disp, vel, co, oc)
    assert _rel(out.disp.cpu().numpy(), rd) < 1e-10
    rng = np.random.default_rng(4)
    dcot, vcot = rng.normal(size=disp.shape), rng.normal(size=disp.shape)
    cot = pb.Particles(conf, ptcl.pmid, torch.from_numpy(dcot).cuda(), torch.from_numpy(vcot).cuda(),
                       torch.zeros_like(out.disp))
    p0, c0, om = run.adjoint(out, cot)
    _, _, rdc, rvc, rom = opm.nbody_adj(pmid, rd, rv, ra, dcot, vcot, np.zeros_like(dcot), co, oc)
    assert _rel(c0.disp.cpu().numpy(), rdc) < 1e-10
    assert _rel(c0.vel.cpu().numpy(), rvc) < 1e-10
    np.testing.assert_allclose(om, rom, rtol=1e-5)
    # the reverse sweep rebuilds the initial state to float64 round-off
    assert _rel(p0.disp.cpu().numpy(), disp) < 1e-12
    # the per-operation adjoints stepped by hand give the same cotangents
    p, c, omi = out, cot, 0.0
    for a_prev, a_next in list(zip(a[:-1], a[1:]))[::-1]:
        p, c, omi, _ = pb.integrate_adj(a_prev, a_next, p, c, cos, omi, conf)
    p, c, om_f, _ = pb.force_adj(float(a[0]), p, c, cos, conf)
    omi += om_f
    assert _rel(c.disp.cpu().numpy(), c0.disp.cpu().numpy()) < 1e-13
    assert _rel(c.vel.cpu().numpy(), c0.vel.cpu().numpy()) < 1e-13
    np.testing.assert_allclose(omi, om, rtol=1e-12)


def test_reverse_sweep_float64_finite_differences():
    a = np.linspace(0.1, 1.0, 4)
    pb, co, conf = _confs(6, 2, a, spacing=8.0)
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    pmid, disp, vel, ptcl = _state(co, conf, pb, 1, 1.0, 0.3)
    rng = np.random.default_rng(7)
    dcot, vcot = rng.normal(size=disp.shape), rng.normal(size=disp.shape)
    u = rng.normal(size=disp.shape)
    u /= np.linalg.norm(u)
    run = pb.NBodyRun(conf, cos)

    def L(d):
        p = pb.Particles(conf, ptcl.pmid, torch.from_numpy(d).cuda(), ptcl.vel)
        o = run.forward(p)
        return float((o.disp.cpu().numpy() * dcot).sum() + (o.vel.cpu().numpy() * vcot).sum())

    eps = 1e-4
    fd = (-L(disp + 2 * eps * u) + 8 * L(disp + eps * u) - 8 * L(disp - eps * u) + L(disp - 2 * eps * u)) / (12 * eps)
    out = run.forward(ptcl)
    cot = pb.Particles(conf, ptcl.pmid, torch.from_numpy(dcot).cuda(), torch.from_numpy(vcot).cuda(),
                       torch.zeros_like(out.disp))
    _, c0, _ = run.adjoint(out, cot)
    np.testing.assert_allclose(float((c0.disp.cpu().numpy() * u).sum()), fd, rtol=1e-6)


def _mode_fd(f, x, u, eps):
    return (-f(x + 2 * eps * u) + 8 * f(x + eps * u) - 8 * f(x - eps * u) + f(x - 2 * eps * u)) / (12 * eps)


def _cdot(g, u):
    """Directional derivative from the packed dL/dRe + i dL/dIm gradient."""
    return float((g.real * u.real).sum() + (g.imag * u.imag).sum())


@pytest.mark.parametrize("order", [1, 2])
def test_lpt_adjoint_float64_finite_differences(order):
    import pmpp_b200 as pb
    from pmpp_b200 import lpt as plpt
    conf = pb.Configuration(4.0, (16, 16, 16), 2, a_start=0.1, float_dtype="float64", lpt_order=order,
                            device="cuda")
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    lin = pb.linear_modes(pb.white_noise_nested(1, conf), cos, conf)
    rng = np.random.default_rng(3)
    n = conf.ptcl_num
    dcot = torch.from_numpy(rng.normal(size=(n, 3))).cuda()
    vcot = torch.from_numpy(rng.normal(size=(n, 3))).cuda()
    res = plpt.lpt_full(lin, cos, conf)
    g, _ = plpt.lpt_vjp(res, dcot, vcot, cos, conf)
    assert g.dtype == torch.complex128
    u = torch.from_numpy(rng.normal(size=lin.shape) + 1j * rng.normal(size=lin.shape)).cuda()
    u = u * (lin.abs().max() / u.abs().max())

    def L(m):
        p = plpt.lpt(m, cos, conf)
        return float((p.disp * dcot).sum() + (p.vel * vcot).sum())

    fd = _mode_fd(L, lin, u, 1e-3)
    np.testing.assert_allclose(_cdot(g, u), fd, rtol=1e-9)


def test_density_loss_gradient_float64_finite_differences():
    import pmpp_b200 as pb
    from pmpp_b200 import lpt as plpt
    from pmpp_b200 import modes as pmodes
    a = np.linspace(0.1, 0.5, 3)
    conf = pb.Configuration(8.0, (8, 8, 8), 2, a_start=0.1, a_custom=a, float_dtype="float64", device="cuda")
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    omega = pb.white_noise_nested(2, conf)
    amp = pmodes.linear_amplitude(cos, conf)
    rng = np.random.default_rng(5)
    target = torch.from_numpy(rng.normal(1.0, 0.3, size=conf.mesh_shape)).cuda()
    run = pb.NBodyRun(conf, cos)

    def forward(w):
        res = plpt.lpt_full(pb.linear_modes(w, cos, conf), cos, conf)
        out = run.forward(res.ptcl)
        return res, out, pb.scatter(out, conf)

    def L(w):
        return float(((forward(w)[2] - target)**2).sum())

    res, out, rho = forward(omega)
    dc, _ = pb.cic.scatter_vjp(out, conf, 2 * (rho - target))
    z = torch.zeros_like(dc)
    _, c0, _ = run.adjoint(out, pb.Particles(conf, out.pmid, dc, z, z.clone()))
    g, _ = plpt.lpt_vjp(res, c0.disp, c0.vel, cos, conf, amp=amp)
    u = torch.from_numpy(rng.normal(size=omega.shape) + 1j * rng.normal(size=omega.shape)).cuda()
    fd = _mode_fd(L, omega, u, 1e-4)
    np.testing.assert_allclose(_cdot(g, u), fd, rtol=1e-6)


def test_pk_loss_gradient_float64_finite_differences():
    """The float64 P(k) loss (deposit, overdensity, D2Z, shell sums) and its
    displacement cotangent (shell-power adjoint, Z2D, overdensity and deposit
    adjoints) against fourth-order differences (1e-6)."""
    import pmpp_b200 as pb
    from pmpp_b200.power_spectrum import pk_loss
    pb_, co, conf = _confs(16, 2)
    pmid, disp, vel, ptcl = _state(co, conf, pb, 3, 1.5, 0.0)
    k, pk, _ = pb.particles_to_pk(ptcl, conf)
    rng = np.random.default_rng(11)
    target = np.asarray(pk) * rng.uniform(0.5, 1.5, size=len(pk))
    loss, dc = pk_loss(ptcl, conf, target)
    assert dc.dtype == torch.float64 and loss > 0
    # a direction of length 30: the derivative stands far above the run-to-run
    # rounding of the deposit's atomic sums (4e-11 in the difference), and no
    # particle's stencil reaches a mesh node, where the CIC weights kink
    u = rng.normal(size=disp.shape)
    u *= 30.0 / np.linalg.norm(u)

    def L(d):
        p = pb.Particles(conf, ptcl.pmid, torch.from_numpy(d).cuda())
        return pk_loss(p, conf, target, grad=False)[0]

    eps = 1e-5
    fd = (-L(disp + 2 * eps * u) + 8 * L(disp + eps * u) - 8 * L(disp - eps * u) + L(disp - 2 * eps * u)) / (12 * eps)
    np.testing.assert_allclose(float((dc.cpu().numpy() * u).sum()), fd, rtol=1e-6)


def test_pk_loss_modes_gradient_float64_finite_differences():
    """The float64 forward model's P(k)-loss gradient w.r.t. the white-noise
    modes (ForwardModel.loss + backward: 2LPT, two KDK steps, the P(k) loss)
    against differences (1e-6)."""
    import pmpp_b200 as pb
    from pmpp_b200 import pipeline
    a = np.linspace(0.1, 0.5, 3)
    conf = pb.Configuration(8.0, (8, 8, 8), 2, a_start=0.1, a_custom=a, float_dtype="float64", device="cuda")
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    omega = pb.white_noise_nested(4, conf)
    model = pipeline.ForwardModel(conf, cos)
    model.forward(omega)
    _, pk0, _ = pb.particles_to_pk(model.final, conf)
    rng = np.random.default_rng(12)
    target = np.asarray(pk0) * rng.uniform(0.6, 1.4, size=len(pk0))
    loss, dc = model.loss(target)
    g = model.backward(dc)["modes"]

    def L(w):
        model.forward(w)
        return model.loss(target, grad=False)[0]

    u = torch.from_numpy(rng.normal(size=omega.shape) + 1j * rng.normal(size=omega.shape)).cuda()
    # step 1e-5: at 1e-4 the difference's own truncation error is about 2e-4 relative
    np.testing.assert_allclose(_cdot(g, u), _mode_fd(L, omega, u, 1e-5), rtol=1e-6)


def test_cosmology_gradients_float64_finite_differences():
    """The float64 forward model's P(k)-loss gradients w.r.t. Omega_m (at fixed
    A_s; growth factors, LPT, force and the linear modes' transfer function) and
    A_s_1e9 against fourth-order differences of the same float64 model with the
    cosmology tables rebuilt at each shifted parameter."""
    import pmpp_b200 as pb
    from pmpp_b200 import pipeline
    a = np.linspace(0.1, 0.5, 3)
    conf = pb.Configuration(8.0, (8, 8, 8), 2, a_start=0.1, a_custom=a, float_dtype="float64", device="cuda")
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    omega = pb.white_noise_nested(4, conf)
    model = pipeline.ForwardModel(conf, cos)
    model.forward(omega)
    _, pk0, _ = pb.particles_to_pk(model.final, conf)
    rng = np.random.default_rng(13)
    target = np.asarray(pk0) * rng.uniform(0.6, 1.4, size=len(pk0))
    _, dc = model.loss(target)
    g = model.backward(dc)

    def L(**kw):
        m = pipeline.ForwardModel(conf, pb.boltzmann(cos.replace(**kw)))
        m.forward(omega)
        return m.loss(target, grad=False)[0]

    def fd(name, x, h):
        return (-L(**{name: x + 2 * h}) + 8 * L(**{name: x + h}) - 8 * L(**{name: x - h})
                + L(**{name: x - 2 * h})) / (12 * h)

    # A_s enters as sqrt(A_s) only: measured 1e-12 apart
    np.testing.assert_allclose(g["A_s_1e9"], fd("A_s_1e9", cos.A_s_1e9, 1e-4), rtol=1e-8)
    # Omega_m: measured 1.2e-6 apart at step 1e-4; the adaptive growth solver's
    # tolerance bounds the difference's own accuracy (1e-5 at step 1e-5, 2e-3
    # truncation at step 1e-3)
    np.testing.assert_allclose(g["Omega_m"], fd("Omega_m", cos.Omega_m, 1e-4), rtol=1e-5)


_PGD = dict(alpha0=0.3, A=0.4, B=0.1, kl=0.1, ks=1.0)


def _oracle_kernel(model, corr, co, a):
    T = {"pm_window": lambda: opm.window_gain(co), "pgd": lambda: opm.pgd_transfer(co, a, **_PGD),
         "softening": lambda: opm.softening_transfer(co, 0.6, 0.5, 1.0),
         "windowed_pgd": lambda: opm.window_gain(co) * opm.pgd_transfer(co, a, **_PGD),
         "pm_window+softening": lambda: opm.window_gain(co) * opm.softening_transfer(co, 0.6, 0.5, 1.0)}.get(model)
    gk = "discrete_laplacian" if corr.green_kernel == 1 else "continuum"
    return opm.potential_kernel(co, gk, None if T is None else T())


@pytest.mark.parametrize("model", ["pm_window", "fastpm_1_4", "fastpm_3_4", "pgd", "softening", "windowed_pgd",
                                   "pm_window+softening", "pm_window:interlaced", "windowed_pgd:interlaced"])
def test_force_with_analytic_corrections_float64(model):
    """The analytic corrections in the float64 force and its adjoint: the
    window compensation (corrections/window.py:229-265), the discrete
    Laplacian (gravity.py:122-171), FastPM's 4-point gradient
    (gravity.py:355-391), PGD at a = 0.5 (corrections/pgd.py:154-237), high-k
    softening (corrections/softening.py:49-80), their products and the
    interlaced deposit (gravity.py:440-463), within 1e-12 of the float64
    oracle (float64 transfer tables, cuFFT D2Z / Z2D)."""
    from pmpp_b200.corrections import init_potential_correction
    pb, co, conf = _confs(16, 2)
    pmid, disp, _, ptcl = _state(co, conf, pb, 5, 1.0)
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    a = 0.5
    il = model.endswith(":interlaced")
    model = model.replace(":interlaced", "")
    corr = init_potential_correction(model, strength=0.6, start=0.5, interlacing=il, **_PGD)
    kernel = _oracle_kernel(model, corr, co, a)
    grad = corr.gradient_kernel
    ref = opm.gravity(pmid, disp, co, cos.Omega_m, kernel=kernel, gradient=grad, interlacing=il)
    ac = np.random.default_rng(6).normal(size=disp.shape)
    rdc, rom = opm.gravity_vjp(pmid, disp, co, cos.Omega_m, ac, kernel=kernel, gradient=grad, interlacing=il)
    acc = pb.gravity(a, ptcl, cos, conf, correction=corr)
    dc, om = pb.gravity_vjp(a, ptcl, cos, conf, torch.from_numpy(ac).cuda(), correction=corr)
    assert acc.dtype == torch.float64 and dc.dtype == torch.float64
    assert _rel(acc.cpu().numpy(), ref) < 1e-12
    assert _rel(dc.cpu().numpy(), rdc) < 1e-12
    np.testing.assert_allclose(om, rom, rtol=1e-12)
    assert _rel(acc.cpu().numpy(), opm.gravity(pmid, disp, co, cos.Omega_m)) > 1e-6  # not the plain force
    if il:  # nor the same correction without interlacing
        assert _rel(acc.cpu().numpy(), opm.gravity(pmid, disp, co, cos.Omega_m, kernel=kernel, gradient=grad)) > 1e-6


@pytest.mark.parametrize("il", [False, True])
def test_pgd_windowed_reverse_sweep_float64_matches_oracle(il):
    """Three KDK steps and the reverse sweep with the window compensation times
    the scale-factor dependent PGD transfer, each force at its positions'
    scale factor, plain and interlaced, against the float64 oracle: positions
    and cotangents within 1e-10, the final acceleration within 1e-9, the
    Omega_m cotangent within 1e-5 (as the plain sweep)."""
    from pmpp_b200.corrections import init_potential_correction
    a = np.linspace(0.1, 1.0, 4)
    pb, co, conf = _confs(16, 2, a)
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    oc = opm.boltzmann(ocos.Cosmo(), co)
    pmid, disp, vel, ptcl = _state(co, conf, pb, 3, 1.0)
    corr = init_potential_correction("windowed_pgd", interlacing=il, **_PGD)
    K = lambda s: _oracle_kernel("windowed_pgd", corr, co, s)
    run = pb.NBodyRun(conf, cos, corr)
    out = run.forward(ptcl)
    rd, rv, ra = opm.nbody(pmid, disp, vel, co, oc, K, interlacing=il)
    assert _rel(out.disp.cpu().numpy(), rd) < 1e-10
    # the force at the final positions amplifies their rounding (measured 1.2e-10)
    assert _rel(out.acc.cpu().numpy(), ra) < 1e-9
    rng = np.random.default_rng(4)
    dcot, vcot = rng.normal(size=disp.shape), rng.normal(size=disp.shape)
    cot = pb.Particles(conf, ptcl.pmid, torch.from_numpy(dcot).cuda(), torch.from_numpy(vcot).cuda(),
                       torch.zeros_like(out.disp))
    _, c0, om = run.adjoint(out, cot)
    _, _, rdc, rvc, rom = opm.nbody_adj(pmid, rd, rv, ra, dcot, vcot, np.zeros_like(dcot), co, oc, K,
                                        interlacing=il)
    assert _rel(c0.disp.cpu().numpy(), rdc) < 1e-10
    assert _rel(c0.vel.cpu().numpy(), rvc) < 1e-10
    np.testing.assert_allclose(om, rom, rtol=1e-5)


def test_interlaced_force_float64_non_cubic_mesh():
    """Interlaced window-compensated force and adjoint in float64 on a non-cubic
    mesh (16 x 12 x 20: the phase's mode numbers differ per axis) within 1e-12
    of the oracle; an empty particle set leaves only the uniform source's
    transform rounding in the force meshes (measured 1.8e-17)."""
    import pmpp_b200 as pb
    from pmpp_b200 import x64
    from pmpp_b200.corrections import init_potential_correction
    shape = (8, 6, 10)
    co = opm.Conf(4.0, shape, mesh_shape=2, a_start=0.1, float_dtype=np.float64)
    conf = pb.Configuration(4.0, shape, 2, a_start=0.1, float_dtype="float64", device="cuda")
    pmid, disp, _, ptcl = _state(co, conf, pb, 9, 1.5)
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    corr = init_potential_correction("pm_window", interlacing=True)
    kernel = opm.potential_kernel(co, "discrete_laplacian", opm.window_gain(co))
    ref = opm.gravity(pmid, disp, co, cos.Omega_m, kernel=kernel, interlacing=True)
    ac = np.random.default_rng(10).normal(size=disp.shape)
    rdc, rom = opm.gravity_vjp(pmid, disp, co, cos.Omega_m, ac, kernel=kernel, interlacing=True)
    acc = pb.gravity(1.0, ptcl, cos, conf, correction=corr)
    dc, om = pb.gravity_vjp(1.0, ptcl, cos, conf, torch.from_numpy(ac).cuda(), correction=corr)
    assert _rel(acc.cpu().numpy(), ref) < 1e-12
    assert _rel(dc.cpu().numpy(), rdc) < 1e-12
    np.testing.assert_allclose(om, rom, rtol=1e-12)
    empty_pmid = torch.zeros((0, 3), dtype=torch.int16, device="cuda")
    empty_disp = torch.zeros((0, 3), dtype=torch.float64, device="cuda")
    acc0, F0 = x64.force(empty_pmid, empty_disp, conf, cos.Omega_m, correction=corr, a=1.0, cosmo=cos)
    assert acc0.shape == (0, 3) and float(F0.abs().max()) < 1e-12


def test_corrected_forward_model_gradients_float64_finite_differences():
    """The float64 forward model with the interlaced, PGD-windowed correction:
    the P(k)-loss gradients w.r.t. the white-noise modes (within 1e-6) and
    Omega_m (within 1e-5, step 1e-4 as the plain model) against differences."""
    import pmpp_b200 as pb
    from pmpp_b200 import pipeline
    from pmpp_b200.corrections import init_potential_correction
    a = np.linspace(0.1, 0.5, 3)
    conf = pb.Configuration(8.0, (8, 8, 8), 2, a_start=0.1, a_custom=a, float_dtype="float64", device="cuda")
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    corr = init_potential_correction("windowed_pgd", interlacing=True, **_PGD)
    omega = pb.white_noise_nested(4, conf)
    model = pipeline.ForwardModel(conf, cos, corr)
    model.forward(omega)
    _, pk0, _ = pb.particles_to_pk(model.final, conf)
    rng = np.random.default_rng(14)
    target = np.asarray(pk0) * rng.uniform(0.6, 1.4, size=len(pk0))
    _, dc = model.loss(target)
    g = model.backward(dc)

    def L(w, c=cos):
        m = pipeline.ForwardModel(conf, c, corr)
        m.forward(w)
        return m.loss(target, grad=False)[0]

    u = torch.from_numpy(rng.normal(size=omega.shape) + 1j * rng.normal(size=omega.shape)).cuda()
    np.testing.assert_allclose(_cdot(g["modes"], u), _mode_fd(L, omega, u, 1e-5), rtol=1e-6)
    Lom = lambda om: L(omega, pb.boltzmann(cos.replace(Omega_m=om)))
    h = 1e-4
    fd = (-Lom(cos.Omega_m + 2 * h) + 8 * Lom(cos.Omega_m + h) - 8 * Lom(cos.Omega_m - h)
          + Lom(cos.Omega_m - 2 * h)) / (12 * h)
    np.testing.assert_allclose(g["Omega_m"], fd, rtol=1e-5)
