"""GPU parity of the hand-written PM FFT passes (pmfft.cu).

Bars: the forward pass chain (z R2C, y, x) against numpy.fft.rfftn in float64
within 1e-5 of the spectrum maximum; the inverse chain against
numpy.fft.irfftn (times the cell count), Hermitian and non-Hermitian input,
within 1e-5 of the output maximum; the fused force and its adjoint through the
pass chain against the cuFFT route and against the oracle within 1e-5.
"""
import numpy as np
import pytest
import torch

from oracle import pm as opm
from tests.helpers import random_particles, rel_err

pytestmark = pytest.mark.gpu

BY = 32


def _lib():
    from pmpp_b200 import _lib
    return _lib


def _stream():
    from pmpp_b200.runtime import stream_handle
    return stream_handle(torch.device("cuda"))


def _block(X, nx, ny, nz):
    """numpy half spectrum (nx, ny, nz//2+1) -> blocked complex64 tensor."""
    P = nz // 2 + 8
    pad = np.zeros((nx, ny, P), np.complex64)
    pad[..., : nz // 2 + 1] = X
    t = torch.from_numpy(pad).view(nx, ny // BY, BY, P).permute(1, 0, 2, 3).contiguous()
    return t.cuda().view(-1)


def _unblock(t, nx, ny, nz, nch=1):
    P = nz // 2 + 8
    a = t.view(nch, ny // BY, nx, BY, P).permute(0, 2, 1, 3, 4).reshape(nch, nx, ny, P)
    return a[..., : nz // 2 + 1].cpu().numpy()


def _ri(z):
    return np.stack([z.real, z.imag])


def _forward(x, nx, ny, nz):
    L = _lib()
    C = L.lib().pmb_pmfft_channel_elems(nx, ny, nz)
    a = torch.empty(C, dtype=torch.complex64, device="cuda")
    b = torch.empty_like(a)
    s = _stream()
    L.call("pmb_pmfft_z", nx, ny, nz, 0, 1, x.data_ptr(), a.data_ptr(), s)
    L.call("pmb_pmfft_col", nx, ny, nz, 0, 1, 0, a.data_ptr(), b.data_ptr(), None, 0, None, None, 0, 1.0, s)
    L.call("pmb_pmfft_col", nx, ny, nz, 4, 1, 0, b.data_ptr(), a.data_ptr(), None, 0, None, None, 0, 1.0, s)
    return a


def _inverse(spec, nx, ny, nz):
    L = _lib()
    b = torch.empty_like(spec)
    out = torch.empty((nx, ny, nz), dtype=torch.float32, device="cuda")
    s = _stream()
    L.call("pmb_pmfft_col", nx, ny, nz, 5, 1, 0, spec.data_ptr(), b.data_ptr(), None, 0, None, None, 0, 1.0, s)
    L.call("pmb_pmfft_col", nx, ny, nz, 1, 1, 0, b.data_ptr(), spec.data_ptr(), None, 0, None, None, 0, 1.0, s)
    L.call("pmb_pmfft_z", nx, ny, nz, 1, 1, spec.data_ptr(), out.data_ptr(), s)
    return out


SHAPES = [(64, 128, 256), (128, 64, 128), (128, 128, 128), (256, 256, 512), (1024, 64, 128)]


@pytest.mark.parametrize("shape", SHAPES)
def test_forward_passes_match_numpy(shape):
    nx, ny, nz = shape
    x = np.random.default_rng(nx + ny + nz).normal(size=shape).astype(np.float32)
    got = _unblock(_forward(torch.from_numpy(x).cuda(), nx, ny, nz), nx, ny, nz)[0]
    ref = np.fft.rfftn(x.astype(np.float64))
    assert rel_err(_ri(got), _ri(ref)) < 1e-5
    assert _lib().pmfft_timeouts() == 0


@pytest.mark.parametrize("shape", SHAPES[:4])
@pytest.mark.parametrize("hermitian", [True, False])
def test_inverse_passes_match_numpy(shape, hermitian):
    nx, ny, nz = shape
    rng = np.random.default_rng(7 + nx)
    if hermitian:
        X = np.fft.rfftn(rng.normal(size=shape))
    else:
        X = rng.normal(size=(nx, ny, nz // 2 + 1)) + 1j * rng.normal(size=(nx, ny, nz // 2 + 1))
    got = _inverse(_block(X.astype(np.complex64), nx, ny, nz), nx, ny, nz).cpu().numpy()
    ref = np.fft.irfftn(X, s=shape) * (nx * ny * nz)
    assert rel_err(got, ref) < 1e-5


def test_padding_columns_stay_zero():
    nx, ny, nz = 64, 64, 128
    x = np.random.default_rng(3).normal(size=(nx, ny, nz)).astype(np.float32)
    a = _forward(torch.from_numpy(x).cuda(), nx, ny, nz)
    P = nz // 2 + 8
    pad = a.view(ny // BY, nx, BY, P)[..., nz // 2 + 1:]
    assert float(pad.abs().max()) == 0.0


def _confs(shape, mesh, spacing=4.0):
    import pmpp_b200 as pb
    co = opm.Conf(spacing, shape, mesh_shape=mesh, a_start=0.1)
    c = pb.Configuration(spacing, shape, mesh, a_start=0.1, device="cuda")
    return pb, co, c


@pytest.mark.parametrize("shape,mesh", [((32, 32, 32), 4), ((32, 16, 64), 4), ((64, 64, 64), 2)])
def test_force_pass_chain_matches_cufft_route(shape, mesh):
    pb, co, conf = _confs(shape, mesh)
    assert _lib().pmfft_active(*conf.mesh_shape)
    pmid, disp = random_particles(co, seed=5, spread=2.0)
    ptcl = pb.Particles(conf, torch.from_numpy(pmid).cuda(), torch.from_numpy(disp).cuda())
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    ac = torch.from_numpy(np.random.default_rng(2).normal(size=disp.shape).astype(np.float32)).cuda()
    res = {}
    try:
        for on in (True, False):
            _lib().set_pmfft(on)
            acc = pb.gravity(1.0, ptcl, cos, conf).cpu().numpy()
            dc, om = pb.gravity_vjp(1.0, ptcl, cos, conf, ac)
            res[on] = (acc, dc.cpu().numpy(), om)
    finally:
        _lib().set_pmfft(True)
    assert rel_err(res[True][0], res[False][0]) < 1e-5
    assert rel_err(res[True][1], res[False][1]) < 1e-5
    np.testing.assert_allclose(res[True][2], res[False][2], rtol=1e-5)
    assert _lib().pmfft_timeouts() == 0


def test_force_pass_chain_matches_oracle():
    pb, co, conf = _confs((32, 32, 32), 4)
    pmid, disp = random_particles(co, seed=11, spread=2.0)
    ptcl = pb.Particles(conf, torch.from_numpy(pmid).cuda(), torch.from_numpy(disp).cuda())
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    acc = pb.gravity(1.0, ptcl, cos, conf).cpu().numpy()
    assert rel_err(acc, opm.gravity(pmid, disp, co, 0.3)) < 1e-5
    ac = np.random.default_rng(1).normal(size=disp.shape).astype(np.float32)
    dc, om = pb.gravity_vjp(1.0, ptcl, cos, conf, torch.from_numpy(ac).cuda())
    rdc, rom = opm.gravity_vjp(pmid, disp, co, 0.3, ac)
    assert rel_err(dc.cpu().numpy(), rdc) < 1e-5
    np.testing.assert_allclose(om, rom, rtol=1e-5)


def test_uniform_lattice_zero_force_pass_chain():
    pb, co, conf = _confs((64, 64, 64), 2)
    ptcl = pb.Particles.gen_grid(conf)
    acc = pb.gravity(1.0, ptcl, pb.boltzmann(pb.SimpleLCDM(conf)), conf)
    assert float(acc.abs().max()) < 3e-7
    assert float(acc.double().sum(0).abs().max()) < 2e-5


def test_staged_route_is_bitwise_the_fused_route():
    from pmpp_b200.runtime import StageTimer
    pb, co, conf = _confs((32, 32, 32), 4)
    pmid, disp = random_particles(co, seed=9, spread=2.0)
    ptcl = pb.Particles(conf, torch.from_numpy(pmid).cuda(), torch.from_numpy(disp).cuda())
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    ac = torch.from_numpy(np.random.default_rng(4).normal(size=disp.shape).astype(np.float32)).cuda()
    fused = (pb.gravity(1.0, ptcl, cos, conf), pb.gravity_vjp(1.0, ptcl, cos, conf, ac)[0])
    with StageTimer() as timer:
        staged = (pb.gravity(1.0, ptcl, cos, conf), pb.gravity_vjp(1.0, ptcl, cos, conf, ac)[0])
    assert "fft_x_green" in timer.counts and "fft_x_green_adj" in timer.counts
    for f, s in zip(fused, staged):
        assert torch.equal(f, s)


def test_split_adjoint_x_pass_matches_fused():
    """Mode 8 (x forward + adjoint multiplier) followed by a plain inverse x pass
    equals the fused mode 7."""
    nx, ny, nz = 128, 64, 128
    pb, co, conf = _confs((nx // 2, ny // 2, nz // 2), 2)
    L = _lib()
    C = L.lib().pmb_pmfft_channel_elems(nx, ny, nz)
    s = _stream()
    x = torch.from_numpy(np.random.default_rng(6).normal(size=(2, nx, ny, nz)).astype(np.float32)).cuda()
    a = torch.empty(2 * C, dtype=torch.complex64, device="cuda")
    b = torch.empty_like(a)
    L.call("pmb_pmfft_z", nx, ny, nz, 0, 2, x.data_ptr(), a.data_ptr(), s)
    L.call("pmb_pmfft_col", nx, ny, nz, 0, 2, 0, a.data_ptr(), b.data_ptr(), None, 0, None, None, 0, 1.0, s)
    tab = conf.spectral_tables("mesh", torch.device("cuda"), 0).data_ptr()
    masks = int(conf.has_particle_nyquist_masks)
    fused = torch.empty(C, dtype=torch.complex64, device="cuda")
    tmp = torch.empty_like(fused)
    split = torch.empty_like(fused)
    L.call("pmb_pmfft_col", nx, ny, nz, 7, 1, 0, b.data_ptr(), fused.data_ptr(), tab, masks, None, None, 0, 0.3, s)
    L.call("pmb_pmfft_col", nx, ny, nz, 8, 1, 0, b.data_ptr(), tmp.data_ptr(), tab, masks, None, None, 0, 0.3, s)
    L.call("pmb_pmfft_col", nx, ny, nz, 5, 1, 0, tmp.data_ptr(), split.data_ptr(), None, 0, None, None, 0, 1.0, s)
    f = torch.view_as_real(fused).cpu().numpy()
    g = torch.view_as_real(split).cpu().numpy()
    assert rel_err(g, f) < 1e-5


def _chain(L, nx, ny, nz, src, tab, masks, prune, s):
    """Forward force chain through the per-pass entry points (pmfft_force's
    order) and the adjoint chain (pmfft_force_adjoint's) on the force meshes."""
    C = L.lib().pmb_pmfft_channel_elems(nx, ny, nz)
    pm = torch.full((5 * C,), float("nan"), dtype=torch.complex64, device="cuda")  # garbage where never written
    aq, fp = pm.data_ptr(), pm.data_ptr() + 16 * C
    F = torch.empty((3, nx, ny, nz), dtype=torch.float32, device="cuda")
    L.call("pmb_pmfft_z2", nx, ny, nz, 0, 1, src.data_ptr(), aq, tab, masks, prune, s)
    L.call("pmb_pmfft_col2", nx, ny, nz, 0, 1, 0, aq, fp, tab, masks, None, None, 0, 1.0, prune, s)
    L.call("pmb_pmfft_col2", nx, ny, nz, 6, 1, 0, fp, aq, tab, masks, None, None, 0, 0.7, prune, s)
    L.call("pmb_pmfft_col2", nx, ny, nz, 1, 1, 0, aq, fp, tab, masks, None, None, 0, 1.0, prune, s)
    L.call("pmb_pmfft_col2", nx, ny, nz, 2, 1, 1, aq, fp + 8 * C, tab, masks, None, None, 0, 1.0, prune, s)
    L.call("pmb_pmfft_z2", nx, ny, nz, 1, 3, fp, F.data_ptr(), tab, masks, prune, s)
    pm.fill_(float("nan"))
    a3, bb = pm.data_ptr(), pm.data_ptr() + 24 * C
    out = torch.empty((nx, ny, nz), dtype=torch.float32, device="cuda")
    L.call("pmb_pmfft_z2", nx, ny, nz, 0, 3, F.data_ptr(), a3, tab, masks, prune, s)
    L.call("pmb_pmfft_col2", nx, ny, nz, 0, 1, 0, a3, bb, tab, masks, None, None, 0, 1.0, prune, s)
    L.call("pmb_pmfft_col2", nx, ny, nz, 3, 1, 1, a3, bb + 8 * C, tab, masks, None, None, 0, 1.0, prune, s)
    L.call("pmb_pmfft_col2", nx, ny, nz, 7, 1, 0, bb, a3, tab, masks, None, None, 0, 0.7, prune, s)
    L.call("pmb_pmfft_col2", nx, ny, nz, 1, 1, 0, a3, a3 + 8 * C, tab, masks, None, None, 0, 1.0, prune, s)
    L.call("pmb_pmfft_z2", nx, ny, nz, 1, 1, a3 + 8 * C, out.data_ptr(), tab, masks, prune, s)
    return F, out


@pytest.mark.parametrize("ptcl,mesh", [((32, 64, 64), 2), ((32, 32, 32), 4), ((64, 32, 128), 2)])
def test_pruned_chain_equals_full_chain(ptcl, mesh):
    """The chain pruned to the particle-Nyquist box (intermediate buffers
    filled with NaN, so a read of a skipped part would show) gives the full
    chain's force meshes and adjoint bit for bit, and both match numpy."""
    pb, co, conf = _confs(ptcl, mesh)
    nx, ny, nz = conf.mesh_shape
    L = _lib()
    s = _stream()
    assert conf.has_particle_nyquist_masks
    tab = conf.spectral_tables("mesh", torch.device("cuda"), 0).data_ptr()
    x = np.random.default_rng(8).normal(size=(nx, ny, nz)).astype(np.float32)
    src = torch.from_numpy(x).cuda()
    full = _chain(L, nx, ny, nz, src, tab, 1, 0, s)
    pruned = _chain(L, nx, ny, nz, src, tab, 1, 1, s)
    for f, p in zip(full, pruned):
        assert torch.isfinite(p).all()
        assert torch.equal(f, p)
    # the live box is what the masks keep: numpy restatement of the forward chain
    kx, ky, kz = (np.asarray(k, np.float64) for k in co.kvec)
    m = opm.nyquist_filter(co).astype(np.float64)
    k2 = kx[:, None, None] ** 2 + ky[None, :, None] ** 2 + kz[None, None, :] ** 2
    with np.errstate(divide="ignore"):
        K = np.where(k2 > 0, -0.7 * m / k2, 0.0)
    phi = K * np.fft.rfftn(x.astype(np.float64))
    cs = [np.asarray(c, np.float64) for c in co.neg_ik]
    ref = np.stack([np.fft.irfftn(1j * c * phi, s=(nx, ny, nz)) * nx * ny * nz for c in
                    (cs[0][:, None, None], cs[1][None, :, None], cs[2][None, None, :])])
    assert rel_err(full[0].cpu().numpy(), ref) < 1e-5
    assert _lib().pmfft_timeouts() == 0
