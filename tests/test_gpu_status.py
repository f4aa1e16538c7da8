"""Failure reporting on the GPU without a GPU fault.

* Bounded waits: the poll limit of the staged gathers' and the FFT passes'
  first copy wait is set to 0, so every wait runs out at once; the CTAs drain
  their copies, raise the timeout counters and return, and pmb_device_status
  reports -6 with flag 1.  The limit is restored and the same calls give correct
  results again, with a clean status.
* Bad input, injected on the host: a NaN displacement raises flag 2 in the
  sorted buffer's status word and device-wide (the reference fails closed on
  bad state, core/utils.py:206-231, nbody/integrator.py:22-33), an infinite
  deposit value raises flag 4; the scatter, gather and adjoint given the flagged
  buffer leave their outputs untouched.
"""
import ctypes

import numpy as np
import pytest
import torch

from oracle import pm as opm
from tests.helpers import random_particles, rel_err

pytestmark = pytest.mark.gpu


def _status_clean():
    from pmpp_b200 import _lib
    torch.cuda.synchronize()
    assert _lib.device_status() == 0


def _expect_flags(bits):
    from pmpp_b200 import _lib
    torch.cuda.synchronize()
    v = ctypes.c_uint32()
    st = _lib.lib().pmb_device_status(ctypes.byref(v))
    assert st == -6 and v.value & bits == bits, (st, v.value)
    assert _lib.device_status() == 0  # cleared by the read


def _particles(shape=(32, 32, 32), mesh=2, seed=0):
    import pmpp_b200 as pb
    co = opm.Conf(2.0, shape, mesh_shape=mesh)
    conf = pb.Configuration(2.0, shape, mesh, device="cuda")
    pmid, disp = random_particles(co, seed, 2.0)
    return pb, co, conf, pmid, disp


def test_wait_limit_zero_times_out_staged_gather_and_recovers():
    from pmpp_b200 import _lib
    from pmpp_b200.cic import SortedParticles
    pb, co, conf, pmid, disp = _particles()
    _status_clean()
    sp = SortedParticles(torch.from_numpy(pmid).cuda(), torch.from_numpy(disp).cuda(), conf)
    mesh3 = torch.randn((3, ) + tuple(co.mesh_shape), generator=torch.Generator().manual_seed(1)).cuda()
    _lib.call("pmb_set_gather_staging", 2)
    try:
        _lib.set_wait_limit(0)
        sp.gather(mesh3)
        torch.cuda.synchronize()
        assert _lib.wait_timeouts() > 0
        _expect_flags(1)
        _lib.set_wait_limit(None)
        got = sp.gather(mesh3).cpu().numpy()
    finally:
        _lib.set_wait_limit(None)
        _lib.call("pmb_set_gather_staging", 0)
    _status_clean()
    ref = opm.gather(pmid, disp, co, mesh3.cpu().numpy().astype(np.float64))
    assert rel_err(got, ref) < 1e-6


def test_wait_limit_zero_times_out_fft_pass_and_recovers():
    from pmpp_b200 import _lib
    nx, ny, nz = 64, 64, 128
    L = _lib.lib()
    C = L.pmb_pmfft_channel_elems(nx, ny, nz)
    s = torch.cuda.current_stream().cuda_stream
    x = torch.randn((nx, ny, nz), generator=torch.Generator().manual_seed(2)).cuda()
    a = torch.zeros(C, dtype=torch.complex64, device="cuda")
    _status_clean()
    try:
        _lib.set_wait_limit(0)
        _lib.call("pmb_pmfft_z", nx, ny, nz, 0, 1, x.data_ptr(), a.data_ptr(), s)
        torch.cuda.synchronize()
        cnt = ctypes.c_uint32()
        _lib.check(L.pmb_pmfft_timeouts(ctypes.byref(cnt)), "pmb_pmfft_timeouts")
        assert cnt.value > 0
        _expect_flags(1)
        _lib.set_wait_limit(None)
        _lib.call("pmb_pmfft_z", nx, ny, nz, 0, 1, x.data_ptr(), a.data_ptr(), s)
    finally:
        _lib.set_wait_limit(None)
    _status_clean()
    # the z pass alone: a real-to-complex transform of every z row
    P = nz // 2 + 8
    got = a.view(ny // 32, nx, 32, P).permute(1, 0, 2, 3).reshape(nx, ny, P)[..., : nz // 2 + 1].cpu().numpy()
    ref = np.fft.rfft(x.cpu().numpy().astype(np.float64), axis=2)
    assert np.abs(got - ref).max() < 1e-5 * np.abs(ref).max()


def test_nan_displacement_flags_the_sort_and_leaves_outputs():
    from pmpp_b200 import _lib
    from pmpp_b200.cic import SortedParticles
    pb, co, conf, pmid, disp = _particles(seed=3)
    disp[123, 1] = np.nan
    _status_clean()
    sp = SortedParticles(torch.from_numpy(pmid).cuda(), torch.from_numpy(disp).cuda(), conf)
    nx, ny, nz = co.mesh_shape
    flags = ctypes.c_uint32()
    _lib.call("pmb_sorted_status", sp.buf.data_ptr(), sp.n, nx, ny, nz, ctypes.byref(flags),
              torch.cuda.current_stream().cuda_stream)
    assert flags.value == 2
    rho = torch.full((1, nx, ny, nz), 7.0, device="cuda")
    sp.scatter(out=rho)
    acc = torch.full((sp.n, 3), 7.0, device="cuda")
    sp.gather(torch.zeros((3, nx, ny, nz), device="cuda"), out=acc)
    dc = torch.full((sp.n, 3), 7.0, device="cuda")
    sp.interp_grad(torch.ones((1, nx, ny, nz), device="cuda"), u_const=1.0, disp_cot=dc, accumulate=True)
    torch.cuda.synchronize()
    assert bool((rho == 7.0).all()) and bool((acc == 7.0).all()) and bool((dc == 7.0).all())
    _expect_flags(2)


def test_infinite_value_flags_the_deposit_and_leaves_output():
    from pmpp_b200.cic import SortedParticles
    pb, co, conf, pmid, disp = _particles(seed=4)
    val = np.ones((len(pmid), 3), np.float32)
    val[77, 2] = np.inf
    _status_clean()
    sp = SortedParticles(torch.from_numpy(pmid).cuda(), torch.from_numpy(disp).cuda(), conf)
    nx, ny, nz = co.mesh_shape
    out = torch.full((3, nx, ny, nz), 7.0, device="cuda")
    sp.scatter(val=torch.from_numpy(val).cuda(), channels=3, out=out)
    torch.cuda.synchronize()
    assert bool((out == 7.0).all())
    _expect_flags(4)
    # a finite deposit afterwards is clean
    sp2 = SortedParticles(torch.from_numpy(pmid).cuda(), torch.from_numpy(disp).cuda(), conf)
    sp2.scatter(val=torch.ones((len(pmid), 3), device="cuda"), channels=3, out=out)
    _status_clean()
    assert rel_err(out.cpu().numpy(), opm.scatter(pmid, disp, co, val=np.ones((len(pmid), 3), np.float32))) < 1e-6
