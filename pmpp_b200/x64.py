"""float64 build of the forward path (the reference's jax_enable_x64 runs).

With ``Configuration(..., float_dtype="float64")`` the public functions
``white_noise_nested``, ``linear_modes``, ``lpt``, ``nbody`` /
``NBodyRun.forward``, ``scatter`` and ``particles_to_pk`` route here: the same
operations as the float32 kernels, evaluated in double precision on the
device (cuFFT D2Z / Z2D, double-precision CIC deposit and gather), for parity
with the reference's float64 results.  The hand-written adjoints exist for
the float32 build only.
"""
from __future__ import annotations

import numpy as np
import torch

from ._lib import call, lib
from .particles import Particles
from .runtime import stream_handle, workspace


def is_x64(conf):
    return conf.float_dtype == torch.float64


def white_noise_nested(seed, conf, device=None):
    device = conf.device if device is None else torch.device(device)
    gx, gy, gz = conf.ptcl_grid_shape
    out = torch.empty((gx, gy, gz // 2 + 1), dtype=torch.complex128, device=device)
    call("pmb_white_noise_nested64", int(seed) & 0xFFFFFFFF, gx, gy, gz, out.data_ptr(), stream_handle(device))
    return out


def linear_modes(modes, cosmo, conf):
    """delta(k) = omega(k) sqrt(V P_lin(|k|)) at a = 1 (modes.py:397-454)."""
    dev = modes.device
    gx, gy, gz = conf.ptcl_grid_shape
    modes = modes.to(torch.complex128).contiguous()
    out = torch.empty_like(modes)
    k = torch.from_numpy(np.concatenate(conf.kvec_spacing).astype(np.float64)).to(dev)
    tk = torch.from_numpy(np.ascontiguousarray(conf.transfer_k, dtype=np.float64)).to(dev)
    tt = torch.from_numpy(np.ascontiguousarray(cosmo.transfer, dtype=np.float64)).to(dev)
    call("pmb_linear_modes64", modes.data_ptr(), out.data_ptr(), gx, gy, gz, k.data_ptr(), tk.data_ptr(),
         tt.data_ptr(), int(tk.numel()), float(cosmo.A_s), float(cosmo.n_s), float(cosmo.Omega_m),
         float(cosmo.k_pivot), 1.0, float(conf.box_vol), stream_handle(dev))
    return out


def lpt(modes, cosmo, conf):
    """1LPT/2LPT particles at conf.a_start (lpt.py:337-449), float64."""
    gx, gy, gz = conf.ptcl_grid_shape
    dev = modes.device
    modes = modes.to(torch.complex128).contiguous()
    ptcl = Particles.gen_grid(conf, vel=True, device=dev)
    fac, _ = cosmo.lpt_factors(conf.a_start)
    fields = torch.empty((6, gx, gy, gz), dtype=torch.float64, device=dev)
    ws = workspace(lib().pmb_lpt64_workspace_bytes(gx, gy, gz), dev, "lpt64")
    call("pmb_lpt64", modes.data_ptr(), gx, gy, gz, float(conf.ptcl_spacing), float(conf.ptcl_cell_vol),
         conf.spectral_tables("particle", dev).data_ptr(), int(conf.lpt_order), float(fac[0, 0]), float(fac[0, 2]),
         float(fac[1, 0]), float(fac[1, 2]), ptcl.pmid.data_ptr(), ptcl.disp.data_ptr(), ptcl.vel.data_ptr(),
         len(ptcl), float(conf.cell_size), fields.data_ptr(), ws.data_ptr(), ws.numel(), stream_handle(dev))
    return ptcl


def force(pmid, disp, conf, omega_m, acc=None, force_meshes=None, drift_vel=None, drift=0.0, vel_kick=None, kick=0.0):
    """PM accelerations (gravity.py:786-814) in float64; with drift_vel the
    drift is applied first, with vel_kick the closing half-kick is fused."""
    nx, ny, nz = conf.mesh_shape
    dev = disp.device
    n = pmid.shape[0]
    if acc is None:
        acc = torch.empty((n, 3), dtype=torch.float64, device=dev)
    if force_meshes is None:
        force_meshes = torch.empty((3, nx, ny, nz), dtype=torch.float64, device=dev)
    ws = workspace(lib().pmb_force64_workspace_bytes(nx, ny, nz), dev, "force64")
    call("pmb_force64", pmid.data_ptr(), disp.data_ptr(), None if drift_vel is None else drift_vel.data_ptr(),
         float(drift), n, nx, ny, nz, float(conf.cell_size), float(conf.mesh_size / conf.ptcl_num), 1.5 * float(omega_m),
         conf.spectral_tables("mesh", dev).data_ptr(), int(conf.has_particle_nyquist_masks), force_meshes.data_ptr(),
         acc.data_ptr(), None if vel_kick is None else vel_kick.data_ptr(), float(kick), ws.data_ptr(), ws.numel(),
         stream_handle(dev))
    return acc, force_meshes


def nbody(ptcl, cosmo, conf, a_nbody=None):
    """Kick-drift-kick run (solver.py:253-273) in float64: initial force, then
    per step kick, drift + force, closing kick (fused into the gather)."""
    from .nbody import _schedule
    a = conf.a_nbody if a_nbody is None else np.asarray(a_nbody)
    disp = ptcl.disp.to(torch.float64).clone()
    vel = ptcl.vel.to(torch.float64).clone() if ptcl.vel is not None else torch.zeros_like(disp)
    acc, F = force(ptcl.pmid, disp, conf, cosmo.Omega_m)
    s = stream_handle(disp.device)
    for a_prev, a_next in zip(a[:-1], a[1:]):
        stages = _schedule(a_prev, a_next, conf)
        i = 0
        while i < len(stages):
            st = stages[i]
            if st[0] == "kick":
                call("pmb_axpy64", vel.data_ptr(), acc.data_ptr(), vel.numel(),
                     float(cosmo.kick_factor(st[1], st[2], st[3])), s)
                i += 1
                continue
            D = float(cosmo.drift_factor(st[1], st[2], st[3]))
            kick_f, vk = 0.0, None
            if i + 1 < len(stages) and stages[i + 1][0] == "kick":
                kst = stages[i + 1]
                kick_f, vk = float(cosmo.kick_factor(kst[1], kst[2], kst[3])), vel
                i += 1
            force(ptcl.pmid, disp, conf, cosmo.Omega_m, acc=acc, force_meshes=F, drift_vel=vel, drift=D, vel_kick=vk,
                  kick=kick_f)
            i += 1
    return ptcl.replace(disp=disp, vel=vel, acc=acc)


def scatter(ptcl, conf, val=None):
    """CIC density (cic/scatter.py:315-338) in float64; val defaults to
    mesh_size / ptcl_num."""
    nx, ny, nz = conf.mesh_shape
    dev = ptcl.disp.device
    rho = torch.empty((nx, ny, nz), dtype=torch.float64, device=dev)
    v = float(conf.mesh_size / conf.ptcl_num) if val is None else float(val)
    call("pmb_deposit64", ptcl.pmid.data_ptr(), ptcl.disp.to(torch.float64).contiguous().data_ptr(), len(ptcl), nx, ny,
         nz, float(conf.cell_size), v, rho.data_ptr(), stream_handle(dev))
    return rho


def _sinc_tables64(conf, device):
    nx, ny, nz = conf.mesh_shape
    parts = [np.sinc(np.fft.fftfreq(nx)), np.sinc(np.fft.fftfreq(ny)), np.sinc(np.arange(nz // 2 + 1) / nz)]
    return torch.from_numpy(np.concatenate(parts).astype(np.float64)).to(device)


def density_to_pk(rho, conf, mas_power=2):
    """(k, P(k), nmodes) over integer shells (power_spectrum.py:251-374) in float64."""
    from .power_spectrum import _finalize, num_shells
    nx, ny, nz = conf.mesh_shape
    dev = rho.device
    s = stream_handle(dev)
    rho = rho.to(torch.float64).contiguous()
    tot = torch.zeros(1, dtype=torch.float64, device=dev)
    call("pmb_sum64", rho.data_ptr(), rho.numel(), tot.data_ptr(), s)
    delta = torch.empty_like(rho)
    call("pmb_overdensity64", rho.data_ptr(), delta.data_ptr(), rho.numel(), tot.data_ptr(), s)
    spec = torch.empty((nx, ny, nz // 2 + 1), dtype=torch.complex128, device=dev)
    w = workspace(lib().pmb_fft64_work_bytes(nx, ny, nz, 1), dev, "fft64")
    call("pmb_rfft3_64", nx, ny, nz, 1, delta.data_ptr(), spec.data_ptr(), w.data_ptr(), s)
    ns = num_shells(conf)
    sums = torch.empty(ns, dtype=torch.float64, device=dev)
    call("pmb_pk_shells64", spec.data_ptr(), nx, ny, nz, _sinc_tables64(conf, dev).data_ptr(), mas_power, ns,
         sums.data_ptr(), s)
    return _finalize(sums, conf)


def particles_to_pk(ptcl, conf, mas_power=2):
    return density_to_pk(scatter(ptcl, conf), conf, mas_power)
