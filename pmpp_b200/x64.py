"""float64 build of the forward path (the reference's jax_enable_x64 runs).

With ``Configuration(..., float_dtype="float64")`` the public functions
``white_noise_nested``, ``linear_modes``, ``lpt``, ``nbody`` /
``NBodyRun.forward``, ``scatter`` and ``particles_to_pk`` route here: the same
operations as the float32 kernels, evaluated in double precision on the
device (cuFFT D2Z / Z2D, double-precision CIC deposit and gather), for parity
with the reference's float64 results.  The adjoints of the N-body run, the
force, the LPT displacements, the deposit, the P(k) loss and the linear
modes' cosmology parameters exist here too (``nbody_adj``, ``force_vjp``,
``lpt_vjp``, ``scatter_vjp``, ``pk_loss``, ``linear_modes_param_cotangents``),
and the force takes the analytic corrections, interlaced or not
(``correction_tables``).
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
    return _linear_with(modes.to(torch.complex128).contiguous(), cosmo, conf, cosmo.transfer)


def _linear_with(modes, cosmo, conf, transfer):
    dev = modes.device
    gx, gy, gz = conf.ptcl_grid_shape
    out = torch.empty_like(modes)
    k = torch.from_numpy(np.concatenate(conf.kvec_spacing).astype(np.float64)).to(dev)
    tk = torch.from_numpy(np.ascontiguousarray(conf.transfer_k, dtype=np.float64)).to(dev)
    tt = torch.from_numpy(np.ascontiguousarray(transfer, dtype=np.float64)).to(dev)
    call("pmb_linear_modes64", modes.data_ptr(), out.data_ptr(), gx, gy, gz, k.data_ptr(), tk.data_ptr(),
         tt.data_ptr(), int(tk.numel()), float(cosmo.A_s), float(cosmo.n_s), float(cosmo.Omega_m),
         float(cosmo.k_pivot), 1.0, float(conf.box_vol), stream_handle(dev))
    return out


def linear_modes_param_cotangents(omega, modes_cot, cosmo, conf, h=1e-6):
    """(dL/dA_s_1e9, dL/dOmega_m) of the float64 linear modes at a = 1 given
    their cotangent (modes.py:397-454 differentiated).

    The modes scale as sqrt(A_s), so dL/dA_s = <cot, lin> / (2 A_s).  They are
    linear in the interpolated transfer function T and carry an explicit
    1/Omega_m, so dL/dOmega_m = <cot, lin(T + e dT) - lin(T - e dT)> / (2e)
    - <cot, lin> / Omega_m with dT = dT/dOmega_m, a central difference of the
    host's FP64 transfer fit; e keeps T - e dT positive, where the kernel's
    sqrt(T^2) is linear."""
    from .cosmology import transfer_fit
    omega = omega.to(torch.complex128).contiguous()
    mc = torch.view_as_real(modes_cot.to(torch.complex128).contiguous())
    s = stream_handle(omega.device)
    n2 = 2 * omega.numel()
    dots = torch.zeros(3, dtype=torch.float64, device=omega.device)
    T = np.asarray(cosmo.transfer, np.float64)
    Tp = transfer_fit(conf.transfer_k, cosmo.replace(Omega_m=cosmo.Omega_m + h), conf)
    Tm = transfer_fit(conf.transfer_k, cosmo.replace(Omega_m=cosmo.Omega_m - h), conf)
    dT = (np.asarray(Tp, np.float64) - np.asarray(Tm, np.float64)) / (2 * h)
    eps = 1e-2
    while np.any(T[1:] - eps * np.abs(dT[1:]) <= 0):
        eps *= 0.5
    for i, tab in enumerate((T, T + eps * dT, T - eps * dT)):
        lin = torch.view_as_real(_linear_with(omega, cosmo, conf, tab))
        call("pmb_dot64", mc.data_ptr(), lin.data_ptr(), n2, dots[i:].data_ptr(), s)
    d = dots.cpu().numpy()
    return float(d[0] / (2 * cosmo.A_s_1e9)), float((d[1] - d[2]) / (2 * eps) - d[0] / cosmo.Omega_m)


def linear_amplitude(cosmo, conf, device=None):
    """sqrt(V P_lin(|k|)) per rFFT cell at a = 1, float64: the linear-mode
    kernel applied to unit modes."""
    device = conf.device if device is None else torch.device(device)
    gx, gy, gz = conf.ptcl_grid_shape
    ones = torch.ones((gx, gy, gz // 2 + 1), dtype=torch.complex128, device=device)
    return linear_modes(ones, cosmo, conf).real.contiguous()


def lpt_full(modes, cosmo, conf):
    """lpt() that also keeps what the adjoint needs (LPTResult: sampled
    gradient fields, each particle's Lagrangian grid cell, growth factors)."""
    from .lpt import LPTResult
    gx, gy, gz = conf.ptcl_grid_shape
    dev = modes.device
    modes = modes.to(torch.complex128).contiguous()
    ptcl = Particles.gen_grid(conf, vel=True, device=dev)
    fac, dfac = cosmo.lpt_factors(conf.a_start)
    fields = torch.empty((6, gx, gy, gz), dtype=torch.float64, device=dev)
    index = torch.empty(len(ptcl), dtype=torch.int64, device=dev)
    ws = workspace(lib().pmb_lpt64_workspace_bytes(gx, gy, gz), dev, "lpt64")
    call("pmb_lpt64_ex", modes.data_ptr(), gx, gy, gz, float(conf.ptcl_spacing), float(conf.ptcl_cell_vol),
         conf.spectral_tables("particle", dev).data_ptr(), int(conf.lpt_order), float(fac[0, 0]), float(fac[0, 2]),
         float(fac[1, 0]), float(fac[1, 2]), ptcl.pmid.data_ptr(), ptcl.disp.data_ptr(), ptcl.vel.data_ptr(),
         len(ptcl), float(conf.cell_size), fields.data_ptr(), index.data_ptr(), ws.data_ptr(), ws.numel(),
         stream_handle(dev))
    return LPTResult(ptcl, modes, fields, index, fac, dfac)


def lpt_vjp(res, disp_cot, vel_cot, cosmo, conf, amp=None):
    """float64 adjoint of lpt (pmb_lpt_vjp64): (modes_cot in the packed
    dL/dRe + i dL/dIm convention, Omega_m cotangent of the growth factors);
    with amp (float64) the cotangent is w.r.t. the white-noise modes."""
    gx, gy, gz = conf.ptcl_grid_shape
    dev = res.modes.device
    order = int(conf.lpt_order)
    fac = res.factors
    mc = torch.empty_like(res.modes)
    if order == 0:
        mc.zero_()
        return mc, 0.0
    dots = torch.zeros(4, dtype=torch.float64, device=dev)
    ws = workspace(lib().pmb_lpt_vjp64_workspace_bytes(gx, gy, gz), dev, "lpt_vjp64")
    dcot = disp_cot.to(torch.float64).contiguous()
    vcot = vel_cot.to(torch.float64).contiguous()
    amp = None if amp is None else amp.to(torch.float64).contiguous()
    call("pmb_lpt_vjp64", res.modes.data_ptr(), gx, gy, gz, float(conf.ptcl_cell_vol),
         conf.spectral_tables("particle", dev).data_ptr(), order, float(fac[0, 0]), float(fac[0, 2]), float(fac[1, 0]),
         float(fac[1, 2]), res.index.data_ptr(), res.fields.data_ptr(), dcot.data_ptr(), vcot.data_ptr(),
         res.index.numel(), None if amp is None else amp.data_ptr(), mc.data_ptr(), dots.data_ptr(), ws.data_ptr(),
         ws.numel(), stream_handle(dev))
    d = dots.cpu().numpy()
    dfac = res.dfactors
    om = sum(dfac[m, 0] * d[2 * m] + dfac[m, 2] * d[2 * m + 1] for m in range(order))
    return mc, float(om)


def scatter_vjp(ptcl, conf, mesh_cot, val=None):
    """float64 adjoint of the constant-value deposit: (disp_cot, val_cot), val_cot
    = sum(mesh_cot * deposit of unit values) (cic/scatter.py:386-437)."""
    nx, ny, nz = conf.mesh_shape
    dev = ptcl.disp.device
    v = float(conf.mesh_size / conf.ptcl_num) if val is None else float(val)
    mc = mesh_cot.to(torch.float64).contiguous()
    disp = ptcl.disp.to(torch.float64).contiguous()
    dc = torch.zeros_like(disp)
    s = stream_handle(dev)
    call("pmb_scatter_vjp64", ptcl.pmid.data_ptr(), disp.data_ptr(), len(ptcl), nx, ny, nz, float(conf.cell_size), v,
         mc.data_ptr(), dc.data_ptr(), s)
    unit = scatter(ptcl, conf, 1.0)
    tot = torch.zeros(1, dtype=torch.float64, device=dev)
    call("pmb_dot64", mc.data_ptr(), unit.data_ptr(), mc.numel(), tot.data_ptr(), s)
    return dc, float(tot.item())


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


def correction_tables(conf, dev, correction=None, a=None, cosmo=None):
    """(spectral tables, float64 transfer or None, interlaced) of the force for
    a correction: the analytic ones (window compensation, FastPM's Green's
    functions and 4-point gradient, PGD, high-k softening and their products,
    corrections/core.py:40-151, 333-334, 396-422), interlaced when the
    correction asks for it (corrections/core.py:381-393).  The mesh CNN and
    the learned radial transfer are float32 only."""
    if correction is None:
        return conf.spectral_tables("mesh", dev), None, False
    from .gravity import _correction_args, _tables, mesh_cnn_of, uses_interlacing
    if mesh_cnn_of(correction) is not None:
        raise NotImplementedError("the float64 build takes no mesh-CNN correction")
    gk, transfer, radial, _ = _correction_args(correction, a, cosmo, conf)
    if radial is not None:
        raise NotImplementedError("the float64 build takes no learned radial transfer")
    if transfer is not None:
        if transfer.dtype != torch.float64:
            raise TypeError("the float64 force needs a float64 transfer table")
        transfer = transfer.to(dev).contiguous()
    return _tables(conf, dev, gk, correction), transfer, bool(uses_interlacing(correction))


def force(pmid, disp, conf, omega_m, acc=None, force_meshes=None, drift_vel=None, drift=0.0, vel_kick=None, kick=0.0,
          correction=None, a=None, cosmo=None):
    """PM accelerations (gravity.py:786-814) in float64; with drift_vel the
    drift is applied first, with vel_kick the closing half-kick is fused; an
    analytic correction at scale factor a (correction_tables)."""
    nx, ny, nz = conf.mesh_shape
    dev = disp.device
    n = pmid.shape[0]
    if acc is None:
        acc = torch.empty((n, 3), dtype=torch.float64, device=dev)
    if force_meshes is None:
        force_meshes = torch.empty((3, nx, ny, nz), dtype=torch.float64, device=dev)
    tables, transfer, il = correction_tables(conf, dev, correction, a, cosmo)
    entry = "pmb_force64_interlaced" if il else "pmb_force64"
    ws = workspace(getattr(lib(), entry + "_workspace_bytes")(nx, ny, nz), dev, "force64")
    call(entry, pmid.data_ptr(), disp.data_ptr(), None if drift_vel is None else drift_vel.data_ptr(),
         float(drift), n, nx, ny, nz, float(conf.cell_size), float(conf.mesh_size / conf.ptcl_num), 1.5 * float(omega_m),
         tables.data_ptr(), int(conf.has_particle_nyquist_masks), None if transfer is None else transfer.data_ptr(),
         force_meshes.data_ptr(), acc.data_ptr(), None if vel_kick is None else vel_kick.data_ptr(), float(kick),
         ws.data_ptr(), ws.numel(), stream_handle(dev))
    return acc, force_meshes


def force_vjp(pmid, disp, conf, omega_m, force_meshes, acc_cot, disp_cot=None, correction=None, a=None, cosmo=None):
    """disp_cot (+)= (d acc / d disp)^T acc_cot in float64 (pmb_force_vjp64),
    force_meshes being force()'s at these positions (same correction and a)."""
    nx, ny, nz = conf.mesh_shape
    dev = disp.device
    n = pmid.shape[0]
    if disp_cot is None:
        disp_cot = torch.zeros((n, 3), dtype=torch.float64, device=dev)
    acc_cot = acc_cot.to(torch.float64).contiguous()
    tables, transfer, il = correction_tables(conf, dev, correction, a, cosmo)
    entry = "pmb_force_vjp64_interlaced" if il else "pmb_force_vjp64"
    ws = workspace(getattr(lib(), entry + "_workspace_bytes")(nx, ny, nz), dev, "force_vjp64")
    call(entry, pmid.data_ptr(), disp.data_ptr(), n, nx, ny, nz, float(conf.cell_size),
         float(conf.mesh_size / conf.ptcl_num), 1.5 * float(omega_m), tables.data_ptr(),
         int(conf.has_particle_nyquist_masks), None if transfer is None else transfer.data_ptr(),
         force_meshes.data_ptr(), acc_cot.data_ptr(), disp_cot.data_ptr(), ws.data_ptr(), ws.numel(),
         stream_handle(dev))
    return disp_cot


def dot(a, b, out, slot):
    """out[slot] += sum a * b (float64, on the device)."""
    call("pmb_dot64", a.data_ptr(), b.data_ptr(), a.numel(), out[slot:].data_ptr(), stream_handle(a.device))


def axpy(y, x, f):
    """y += x * f in place (two roundings, as the reference's update)."""
    call("pmb_axpy64", y.data_ptr(), x.data_ptr(), y.numel(), float(f), stream_handle(y.device))


def nbody_adj(ptcl, ptcl_cot, cosmo, conf, a_nbody=None, force_meshes=None, correction=None):
    """Reverse sweep in float64 (nbody/solver.py:385-444; integrator.py:429-509,
    541-582, 620-686, 781-837), stage by stage: a kick adjoint restores vel
    and moves vel_cot into acc_cot; a drift stage takes the force adjoint at
    the current positions, restores disp, moves disp_cot into vel_cot and
    recomputes the acceleration there.  The Omega_m cotangent sums the time
    factors' derivatives times their dots and, per force, sum(acc_cot acc) /
    Omega_m (the force is linear in Omega_m).  force_meshes: force()'s meshes
    at ptcl's positions (recomputed when None).  An analytic correction
    enters every force at its positions' scale factor (correction_tables).
    Returns (ptcl_in, ptcl_cot_in, Omega_m_cot)."""
    from .nbody import _schedule
    a = conf.a_nbody if a_nbody is None else np.asarray(a_nbody)
    f64 = lambda t: t.to(torch.float64).clone().contiguous()
    pmid = ptcl.pmid
    disp, vel = f64(ptcl.disp), f64(ptcl.vel)
    dev = disp.device
    z = torch.zeros_like(disp)
    dc = f64(ptcl_cot.disp) if ptcl_cot.disp is not None else z.clone()
    vc = f64(ptcl_cot.vel) if ptcl_cot.vel is not None else z.clone()
    ac = f64(ptcl_cot.acc) if ptcl_cot.acc is not None else z.clone()
    kw = dict(correction=correction, cosmo=cosmo)
    if force_meshes is None or ptcl.acc is None:
        acc, F = force(pmid, disp, conf, cosmo.Omega_m, a=float(a[-1]), **kw)
    else:
        acc, F = f64(ptcl.acc), force_meshes
    stages = []
    for a_prev, a_next in zip(a[:-1][::-1], a[1:][::-1]):
        stages.extend(reversed(_schedule(a_prev, a_next, conf)))
    dots = torch.zeros(3 * len(stages) + 1, dtype=torch.float64, device=dev)
    grads, force_slots, slot = [], [], 0
    for st in stages:
        if st[0] == "kick":
            K, dK = cosmo.kick_factor(st[1], st[2], st[3], with_grad=True)
            dot(vc, acc, dots, slot)
            grads.append((dK, slot))
            slot += 1
            axpy(vel, acc, -K)
            axpy(ac, vc, K)
            continue
        _, a_vel, a_dp, a_dn, a_acc_in = st
        dot(ac, acc, dots, slot)
        force_slots.append(slot)
        slot += 1
        force_vjp(pmid, disp, conf, cosmo.Omega_m, F, ac, dc, a=float(a_dn), **kw)
        ac.zero_()
        D, dD = cosmo.drift_factor(a_vel, a_dp, a_dn, with_grad=True)
        axpy(disp, vel, -D)
        axpy(vc, dc, D)
        dot(dc, vel, dots, slot)
        grads.append((dD, slot))
        slot += 1
        acc, F = force(pmid, disp, conf, cosmo.Omega_m, acc=acc, force_meshes=F, a=float(a_dp), **kw)
    dot(ac, acc, dots, slot)
    force_slots.append(slot)
    force_vjp(pmid, disp, conf, cosmo.Omega_m, F, ac, dc, a=float(a[0]), **kw)
    ac.zero_()
    d = dots.cpu().numpy()
    om = sum(g * d[k] for g, k in grads) + sum(d[k] for k in force_slots) / float(cosmo.Omega_m)
    from .particles import Particles
    return (ptcl.replace(disp=disp, vel=vel, acc=acc), Particles(conf, pmid, dc, vc, ac), float(om))


def nbody(ptcl, cosmo, conf, a_nbody=None, correction=None):
    """Kick-drift-kick run (solver.py:253-273) in float64: initial force, then
    per step kick, drift + force, closing kick (fused into the gather); an
    analytic correction at each force's scale factor."""
    from .nbody import _schedule
    a = conf.a_nbody if a_nbody is None else np.asarray(a_nbody)
    disp = ptcl.disp.to(torch.float64).clone()
    vel = ptcl.vel.to(torch.float64).clone() if ptcl.vel is not None else torch.zeros_like(disp)
    kw = dict(correction=correction, cosmo=cosmo)
    acc, F = force(ptcl.pmid, disp, conf, cosmo.Omega_m, a=float(a[0]), **kw)
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
                  kick=kick_f, a=float(st[3]), **kw)
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


def pk_loss(ptcl, conf, pk_target, mas_power=2, grad=True, kmax=None):
    """The P(k) loss of power_spectrum.pk_loss in float64 (deposit, overdensity,
    D2Z, shell sums) and its displacement cotangent through the transposed
    stages: shell-power adjoint, Z2D, the overdensity's adjoint (the mean
    included) and the deposit's position term (cic/scatter.py:386-437)."""
    from .power_spectrum import _finalize, num_shells
    nx, ny, nz = conf.mesh_shape
    dev = ptcl.disp.device
    s = stream_handle(dev)
    rho = scatter(ptcl, conf)
    tot = torch.zeros(1, dtype=torch.float64, device=dev)
    call("pmb_sum64", rho.data_ptr(), rho.numel(), tot.data_ptr(), s)
    delta = torch.empty_like(rho)
    call("pmb_overdensity64", rho.data_ptr(), delta.data_ptr(), rho.numel(), tot.data_ptr(), s)
    spec = torch.empty((nx, ny, nz // 2 + 1), dtype=torch.complex128, device=dev)
    w = workspace(lib().pmb_fft64_work_bytes(nx, ny, nz, 1), dev, "fft64")
    call("pmb_rfft3_64", nx, ny, nz, 1, delta.data_ptr(), spec.data_ptr(), w.data_ptr(), s)
    ns = num_shells(conf)
    sinc = _sinc_tables64(conf, dev)
    sums = torch.empty(ns, dtype=torch.float64, device=dev)
    call("pmb_pk_shells64", spec.data_ptr(), nx, ny, nz, sinc.data_ptr(), mas_power, ns, sums.data_ptr(), s)
    k, pk, nmodes = _finalize(sums, conf)
    tgt = np.asarray(pk_target, dtype=np.float64)
    valid = (nmodes > 0) & (pk > 0) & (tgt > 0)
    if kmax is not None:
        valid &= k <= kmax
    lr = np.where(valid, np.log(np.where(valid, pk, 1.0) / np.where(valid, tgt, 1.0)), 0.0)
    nv = max(int(valid.sum()), 1)
    loss = float((lr**2).sum() / nv)
    if not grad:
        return loss, None
    norm = conf.cell_size**3 / conf.mesh_size
    wsh = np.zeros(ns)
    wsh[1:] = np.where(valid, 2 * lr / nv / np.where(valid, pk, 1.0), 0.0) * norm / np.maximum(nmodes, 1)
    wd = torch.from_numpy(wsh).to(dev)
    gspec = torch.empty_like(spec)
    call("pmb_pk_shells_adjoint64", spec.data_ptr(), nx, ny, nz, sinc.data_ptr(), mas_power, ns, wd.data_ptr(), 1.0,
         gspec.data_ptr(), s)
    dcot = torch.empty((nx, ny, nz), dtype=torch.float64, device=dev)
    call("pmb_irfft3_64", nx, ny, nz, 1, gspec.data_ptr(), dcot.data_ptr(), w.data_ptr(), s)
    # delta = rho / m - 1 with m = sum(rho)/M:  rho_cot = dcot/m - sum(dcot*rho)/(m^2 M)
    dd = torch.zeros(1, dtype=torch.float64, device=dev)
    call("pmb_dot64", dcot.data_ptr(), rho.data_ptr(), rho.numel(), dd.data_ptr(), s)
    m = float(tot.item()) / rho.numel()
    rho_cot = dcot.mul_(1.0 / m).sub_(float(dd.item()) / (m * m * rho.numel()))
    disp_cot, _ = scatter_vjp(ptcl, conf, rho_cot)
    return loss, disp_cot
