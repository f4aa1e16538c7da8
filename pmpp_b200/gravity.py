"""Particle-mesh gravity and its adjoint (nbody/gravity.py:786-814).

acc = gather(irfft((i c_d) K(k) rfft((rho - 1) * 1.5 Omega_m)))  for d = x, y, z
with K = particle-Nyquist mask x Green's function x optional transfer.  The
whole chain runs as one C-ABI call (pmb_force): sort, deterministic scatter
straight into the Poisson source, R2C, fused Green x gradient, one batched
C2R for the three force meshes, and a three-channel gather.

``correction`` accepts None or an object with ``green_kernel`` (0 continuum,
1 discrete Laplacian), ``gradient_kernel`` ("spectral" or "fastpm_4point"),
optionally ``interlacing`` and ``transfer_tables(a, cosmo, conf)`` returning
(transfer half-spectrum tensor or None, radial |n|^2 table or None); see
pmpp_b200/corrections.py.  An interlaced correction takes its own staged
route (two deposits, cuFFT, pmb_interlace_spectra).
"""
from __future__ import annotations

import numpy as np
import torch

from ._lib import call, lib, pmfft_active
from .runtime import StageTimer, ptr, require_cuda, stream_handle, workspace


def _om32(omega_m):
    return float(np.float32(omega_m))


def _lane_suffix(lane):
    """Lane "0" is the default workspace (a forward run's last force doubles as it)."""
    return "" if lane in ("", "0") else lane


def _stage_buffers(n, conf, dev, sorted_lane="", work_lane=""):
    """Workspace views of the staged force and force adjoint.

    sorted_lane names the sorted-record buffer (the reverse sweep alternates
    two so a force adjoint can read one while the next force writes the
    other); work_lane the scratch, meshes and spectra ("v" gives a force
    adjoint its own set, for running beside a force evaluation)."""
    L = lib()
    nx, ny, nz = conf.mesh_shape
    sorted_buf = workspace(L.pmb_sorted_bytes(n, nx, ny, nz), dev, "st_sorted" + _lane_suffix(sorted_lane))
    sort_scr = workspace(L.pmb_sort_scratch_bytes(n, nx, ny, nz), dev, "st_sortscr" + work_lane)
    s16 = workspace(16, dev, "st_s16" + work_lane)
    real3 = workspace(12 * conf.mesh_size, dev, "st_real3" + work_lane)
    return sorted_buf, sort_scr, s16, real3


def _cufft_buffers(conf, dev):
    """Half spectra and cuFFT work area of the cuFFT route."""
    L = lib()
    nx, ny, nz = conf.mesh_shape
    Mc = nx * ny * (nz // 2 + 1)
    spec3 = workspace(24 * Mc, dev, "st_spec3")
    spec1 = workspace(8 * Mc, dev, "st_spec1")
    fw = max(L.pmb_fft_work_bytes(nx, ny, nz, 3), L.pmb_fft_work_bytes(nx, ny, nz, 1))
    work = workspace(fw, dev, "st_fftwork")
    return spec3, spec1, work


def mesh_cnn_of(correction):
    """The mesh-CNN part of a correction (itself, or a combined correction's), or None."""
    if correction is None:
        return None
    if getattr(correction, "mesh_cnn", False):
        return correction
    for c in getattr(correction, "parts", None) or ():
        if getattr(c, "mesh_cnn", False):
            return c
    return None


def _cnn_buffers(conf, dev, lane=""):
    """Two extra half spectra and real meshes of the residual-potential route."""
    L = lib()
    nx, ny, nz = conf.mesh_shape
    Mc = nx * ny * (nz // 2 + 1)
    specA = workspace(8 * Mc, dev, "cnn_specA" + lane)
    specB = workspace(8 * Mc, dev, "cnn_specB" + lane)
    real2 = workspace(8 * conf.mesh_size, dev, "cnn_real2" + lane)
    return specA, specB, real2


def _cnn_potential_and_residual(pmid, disp, conf, omega_m, tables, gk, transfer, radial, rl, sorted_buf, s16, real3,
                                spec1, specA, work, cnn, a, cosmo, keep, s):
    """S (real3[0]), its spectrum (spec1), phi = irfft(K S_hat) (real3[1]) and
    the residual R of the mesh CNN (corrections/core.py:321-331)."""
    n = pmid.shape[0]
    nx, ny, nz = conf.mesh_shape
    M = conf.mesh_size
    masks = int(conf.has_particle_nyquist_masks)
    call("pmb_scatter_rows", sorted_buf.data_ptr(), n, nx, ny, nz, 1, None, 0, float(conf.mesh_size / conf.ptcl_num),
         1, 1.5 * _om32(omega_m), real3.data_ptr(), s16.data_ptr(), s)
    call("pmb_rfft3", nx, ny, nz, 1, real3.data_ptr(), spec1.data_ptr(), work.data_ptr(), s)
    call("pmb_green_potential", spec1.data_ptr(), specA.data_ptr(), nx, ny, nz, tables.data_ptr(), masks, gk,
         ptr(transfer), ptr(radial), rl, float(1.0 / M), s)
    call("pmb_irfft3", nx, ny, nz, 1, specA.data_ptr(), real3.data_ptr() + 4 * M, work.data_ptr(), s)
    f32 = real3.view(torch.float32)
    S, phi = f32[:M].view(nx, ny, nz), f32[M:2 * M].view(nx, ny, nz)
    return S, phi, cnn.residual(S, phi, a, cosmo, keep=keep)


def _force_cnn(pmid, disp, conf, omega_m, tables, gk, transfer, radial, rl, F, acc, drift_vel, drift, vel_kick, kick,
               kick2, timer, cnn, a, cosmo, lane=""):
    """Force with the mesh-CNN residual potential on the cuFFT route:
    sort, deposit S, R2C, P = K S_hat, phi = C2R(P), R = CNN(S, phi), R2C,
    gradients of P + rfft(R) / cells, three C2R, gather."""
    n = pmid.shape[0]
    nx, ny, nz = conf.mesh_shape
    dev = disp.device
    s = stream_handle(dev)
    M = conf.mesh_size
    sorted_buf, sort_scr, s16, real3 = _stage_buffers(n, conf, dev, sorted_lane=lane)
    spec3, spec1, work = _cufft_buffers(conf, dev)
    specA, specB, _ = _cnn_buffers(conf, dev)
    timer = _NoTimer() if timer is None else timer
    t = timer.start()
    call("pmb_sort_rows", pmid.data_ptr(), disp.data_ptr(), ptr(drift_vel), float(drift), n, nx, ny, nz,
         float(conf.cell_size), sorted_buf.data_ptr(), sort_scr.data_ptr(), sort_scr.numel(), s)
    t = timer.mark("sort", t)
    _, _, R = _cnn_potential_and_residual(pmid, disp, conf, omega_m, tables, gk, transfer, radial, rl, sorted_buf, s16,
                                          real3, spec1, specA, work, cnn, a, cosmo, False, s)
    t = timer.mark("mesh_cnn", t)
    call("pmb_rfft3", nx, ny, nz, 1, R.data_ptr(), specB.data_ptr(), work.data_ptr(), s)
    masks = int(conf.has_particle_nyquist_masks)
    call("pmb_green_potential", spec1.data_ptr(), specA.data_ptr(), nx, ny, nz, tables.data_ptr(), masks, gk,
         ptr(transfer), ptr(radial), rl, float(1.0 / M), s)
    call("pmb_gradient_spectra", specA.data_ptr(), specB.data_ptr(), float(1.0 / M), spec3.data_ptr(), nx, ny, nz,
         tables.data_ptr(), 1.0, s)
    call("pmb_irfft3", nx, ny, nz, 3, spec3.data_ptr(), F.data_ptr(), work.data_ptr(), s)
    t = timer.mark("fft_green_c2r", t)
    call("pmb_gather_rows2", sorted_buf.data_ptr(), n, nx, ny, nz, 3, F.data_ptr(), acc.data_ptr(), ptr(vel_kick),
         float(kick), float(kick2), s)
    timer.mark("gather", t)


def _force_vjp_cnn(pmid, disp, conf, omega_m, tables, gk, transfer, radial, rl, F, acc_cot, disp_cot, timer, cnn, a,
                   cosmo, presorted=False, sorted_lane="", work_lane="", om_out=None):
    """Transpose of _force_cnn.  With H_d = i c_d K and the residual path
    R -> irfft(i c_d rfft(R)) both real convolutions, the source cotangent is
    irfft(conj(H_d) rfft(F_cot)) + dS_R + irfft(K rfft(dphi)), where R_cot =
    irfft(conj(i c_d) rfft(F_cot)) and (dS_R, dphi) come from the network's
    backward; the network's parameter gradients go to cnn.grad.  om_out (a
    list) receives the Omega_m cotangent: sum(S_cot S) / Omega_m plus the
    conditioning feature's."""
    n = pmid.shape[0]
    nx, ny, nz = conf.mesh_shape
    dev = disp.device
    s = stream_handle(dev)
    M = conf.mesh_size
    masks = int(conf.has_particle_nyquist_masks)
    slane = sorted_lane if presorted else work_lane
    sorted_buf, sort_scr, s16, real3 = _stage_buffers(n, conf, dev, slane, work_lane)
    spec3, spec1, work = _cufft_buffers(conf, dev)
    specA, specB, real2 = _cnn_buffers(conf, dev, work_lane)
    timer = _NoTimer() if timer is None else timer
    t = timer.start()
    if not presorted:
        call("pmb_sort_rows", pmid.data_ptr(), disp.data_ptr(), None, 0.0, n, nx, ny, nz, float(conf.cell_size),
             sorted_buf.data_ptr(), sort_scr.data_ptr(), sort_scr.numel(), s)
        t = timer.mark("sort", t)
    cot_sorted = workspace(12 * n, dev, "st_cot_sorted" + work_lane)
    call("pmb_interp_grad_rows", sorted_buf.data_ptr(), n, nx, ny, nz, 3, F.data_ptr(), acc_cot.data_ptr(), 0.0,
         float(conf.cell_size), 1, disp_cot.data_ptr(), None, cot_sorted.data_ptr(), s)
    call("pmb_scatter_rows", sorted_buf.data_ptr(), n, nx, ny, nz, 3, cot_sorted.data_ptr(), 1, 0.0, 0, 1.0,
         real3.data_ptr(), s16.data_ptr(), s)
    call("pmb_rfft3", nx, ny, nz, 3, real3.data_ptr(), spec3.data_ptr(), work.data_ptr(), s)
    # direct path (S_cot1) and residual path (R_cot), both with 1 / cells
    f2 = real2.view(torch.float32)
    Sc, Rc = f2[:M].view(nx, ny, nz), f2[M:2 * M].view(nx, ny, nz)
    call("pmb_green_gradient_adjoint", spec3.data_ptr(), spec1.data_ptr(), nx, ny, nz, tables.data_ptr(), masks, gk,
         ptr(transfer), ptr(radial), rl, float(1.0 / M), s)
    call("pmb_irfft3", nx, ny, nz, 1, spec1.data_ptr(), Sc.data_ptr(), work.data_ptr(), s)
    call("pmb_gradient_adjoint_plain", spec3.data_ptr(), specB.data_ptr(), nx, ny, nz, tables.data_ptr(),
         float(1.0 / M), s)
    call("pmb_irfft3", nx, ny, nz, 1, specB.data_ptr(), Rc.data_ptr(), work.data_ptr(), s)
    t = timer.mark("adjoint_spectral", t)
    # the network at these positions, then its backward
    S, phi, _ = _cnn_potential_and_residual(pmid, disp, conf, omega_m, tables, gk, transfer, radial, rl, sorted_buf,
                                            s16, real3, spec1, specA, work, cnn, a, cosmo, True, s)
    dS, dphi, dparams, dfeat = cnn.residual_adjoint(Rc)
    if cnn.accumulate_grads:
        cnn.grad += dparams
    t = timer.mark("mesh_cnn_adjoint", t)
    # phi = irfft(K rfft(S)) is a real convolution with K even: its transpose is itself
    call("pmb_rfft3", nx, ny, nz, 1, dphi.data_ptr(), specB.data_ptr(), work.data_ptr(), s)
    call("pmb_green_potential", specB.data_ptr(), specA.data_ptr(), nx, ny, nz, tables.data_ptr(), masks, gk,
         ptr(transfer), ptr(radial), rl, float(1.0 / M), s)
    call("pmb_irfft3", nx, ny, nz, 1, specA.data_ptr(), dphi.data_ptr(), work.data_ptr(), s)
    call("pmb_axpy", Sc.data_ptr(), dS.data_ptr(), M, 1.0, s)
    call("pmb_axpy", Sc.data_ptr(), dphi.data_ptr(), M, 1.0, s)
    om32 = _om32(omega_m)
    if om_out is not None:
        d = torch.zeros(1, dtype=torch.float64, device=dev)
        call("pmb_dot", Sc.data_ptr(), S.data_ptr(), M, d.data_ptr(), s)
        om_out.append(float(d.item()) / om32 + float(dfeat[1]))
    call("pmb_interp_grad_rows", sorted_buf.data_ptr(), n, nx, ny, nz, 1, Sc.data_ptr(), None,
         float(conf.mesh_size / conf.ptcl_num) * 1.5 * om32, float(conf.cell_size), 1, disp_cot.data_ptr(), None,
         None, s)
    timer.mark("scatter_adjoint", t)


def uses_interlacing(correction):
    """force_uses_interlacing (corrections/core.py:381-393): a correction, or
    any part of a combined one, asking for interlaced assignment."""
    if correction is None:
        return False
    parts = getattr(correction, "parts", None)
    if parts is not None:
        return any(uses_interlacing(c) for c in parts)
    return bool(getattr(correction, "interlacing", False))


def _interlace_buffers(n, conf, dev, sorted_lane="", work_lane=""):
    """Sorted records at the half-cell-shifted origin, two half spectra, three
    half spectra and the cuFFT work area of the interlaced route."""
    L = lib()
    nx, ny, nz = conf.mesh_shape
    Mc = nx * ny * (nz // 2 + 1)
    sorted_sh = workspace(L.pmb_sorted_bytes(n, nx, ny, nz), dev, "st_sorted_sh" + _lane_suffix(sorted_lane))
    spec2 = workspace(16 * Mc, dev, "il_spec2" + work_lane)
    spec3 = workspace(24 * Mc, dev, "il_spec3" + work_lane)
    fw = max(L.pmb_fft_work_bytes(nx, ny, nz, b) for b in (1, 2, 3))
    work = workspace(fw, dev, "il_fftwork" + work_lane)
    return sorted_sh, spec2, spec3, work


def _sort_both(pmid, disp, conf, drift_vel, drift, sorted_buf, sorted_sh, sort_scr, s):
    """Cell-sorted records at the mesh origin and at (cell/2, cell/2, cell/2)
    (gravity.py:455-457: scatter(..., offset=cell/2)); the drift, when given,
    is applied by the first sort."""
    n = pmid.shape[0]
    nx, ny, nz = conf.mesh_shape
    h = float(conf.cell_size) / 2
    call("pmb_sort_rows", pmid.data_ptr(), disp.data_ptr(), ptr(drift_vel), float(drift), n, nx, ny, nz,
         float(conf.cell_size), sorted_buf.data_ptr(), sort_scr.data_ptr(), sort_scr.numel(), s)
    call("pmb_sort_rows_ex", pmid.data_ptr(), disp.data_ptr(), None, 0.0, n, nx, ny, nz, float(conf.cell_size), h, h,
         h, None, sorted_sh.data_ptr(), sort_scr.data_ptr(), sort_scr.numel(), s)


def _force_interlaced(pmid, disp, conf, omega_m, tables, gk, transfer, radial, rl, F, acc, drift_vel, drift, vel_kick,
                      kick, kick2, timer, src_hat_out=None, lane=""):
    """Interlaced force (gravity.py:446-463, 809-811): the regular and the
    half-cell-shifted deposits, one batched R2C of both, the phase-shifted
    average (pmb_interlace_spectra), then Green x gradient, three C2R and the
    three-channel gather at the regular origin."""
    n = pmid.shape[0]
    nx, ny, nz = conf.mesh_shape
    dev = disp.device
    s = stream_handle(dev)
    M = conf.mesh_size
    Mc = nx * ny * (nz // 2 + 1)
    sorted_buf, sort_scr, s16, real3 = _stage_buffers(n, conf, dev, sorted_lane=lane)
    sorted_sh, spec2, spec3, work = _interlace_buffers(n, conf, dev, sorted_lane=lane)
    timer = _NoTimer() if timer is None else timer
    t = timer.start()
    _sort_both(pmid, disp, conf, drift_vel, drift, sorted_buf, sorted_sh, sort_scr, s)
    t = timer.mark("sort", t)
    vc = float(conf.mesh_size / conf.ptcl_num)
    for k, sb in enumerate((sorted_buf, sorted_sh)):
        call("pmb_scatter_rows", sb.data_ptr(), n, nx, ny, nz, 1, None, 0, vc, 1, 1.5 * _om32(omega_m),
             real3.data_ptr() + 4 * M * k, s16.data_ptr(), s)
    t = timer.mark("scatter", t)
    call("pmb_rfft3", nx, ny, nz, 2, real3.data_ptr(), spec2.data_ptr(), work.data_ptr(), s)
    t = timer.mark("fft_r2c", t)
    call("pmb_interlace_spectra", spec2.data_ptr(), spec2.data_ptr() + 8 * Mc, nx, ny, nz, 0, s)
    if src_hat_out is not None:
        src_hat_out.view(torch.uint8).view(-1)[:8 * Mc].copy_(spec2[:8 * Mc])
    call("pmb_green_gradient", spec2.data_ptr(), spec3.data_ptr(), nx, ny, nz, tables.data_ptr(),
         int(conf.has_particle_nyquist_masks), gk, ptr(transfer), ptr(radial), rl, float(1.0 / M), s)
    t = timer.mark("green_gradient", t)
    call("pmb_irfft3", nx, ny, nz, 3, spec3.data_ptr(), F.data_ptr(), work.data_ptr(), s)
    t = timer.mark("fft_c2r", t)
    call("pmb_gather_rows2", sorted_buf.data_ptr(), n, nx, ny, nz, 3, F.data_ptr(), acc.data_ptr(), ptr(vel_kick),
         float(kick), float(kick2), s)
    timer.mark("gather", t)


def _force_vjp_interlaced(pmid, disp, conf, omega_m, tables, gk, transfer, radial, rl, F, acc_cot, disp_cot, timer,
                          src_hat=None, transfer_cot_out=None, presorted=False, sorted_lane="", work_lane=""):
    """Transpose of the interlaced force: the gather adjoint, the acceleration
    cotangents deposited, R2C, the adjoint multiplier, the transposed phase
    split (pmb_interlace_spectra mode 1) into the two deposits' cotangent
    spectra, one batched C2R and the deposit adjoints at both origins."""
    n = pmid.shape[0]
    nx, ny, nz = conf.mesh_shape
    dev = disp.device
    s = stream_handle(dev)
    M = conf.mesh_size
    Mc = nx * ny * (nz // 2 + 1)
    slane = sorted_lane if presorted else work_lane
    sorted_buf, sort_scr, s16, real3 = _stage_buffers(n, conf, dev, slane, work_lane)
    sorted_sh, spec2, spec3, work = _interlace_buffers(n, conf, dev, slane, work_lane)
    timer = _NoTimer() if timer is None else timer
    t = timer.start()
    if not presorted:
        _sort_both(pmid, disp, conf, None, 0.0, sorted_buf, sorted_sh, sort_scr, s)
        t = timer.mark("sort", t)
    cot_sorted = workspace(12 * n, dev, "st_cot_sorted" + work_lane)
    call("pmb_interp_grad_rows", sorted_buf.data_ptr(), n, nx, ny, nz, 3, F.data_ptr(), acc_cot.data_ptr(), 0.0,
         float(conf.cell_size), 1, disp_cot.data_ptr(), None, cot_sorted.data_ptr(), s)
    t = timer.mark("gather_adjoint", t)
    call("pmb_scatter_rows", sorted_buf.data_ptr(), n, nx, ny, nz, 3, cot_sorted.data_ptr(), 1, 0.0, 0, 1.0,
         real3.data_ptr(), s16.data_ptr(), s)
    t = timer.mark("scatter3", t)
    masks = int(conf.has_particle_nyquist_masks)
    call("pmb_rfft3", nx, ny, nz, 3, real3.data_ptr(), spec3.data_ptr(), work.data_ptr(), s)
    t = timer.mark("fft_r2c", t)
    if transfer_cot_out is not None:
        call("pmb_transfer_cot", spec3.data_ptr(), src_hat.data_ptr(), nx, ny, nz, tables.data_ptr(), masks,
             int(transfer_cot_out.numel()), transfer_cot_out.data_ptr(), s)
    post = float(np.float32(1.5 * _om32(omega_m)) / M)
    call("pmb_green_gradient_adjoint", spec3.data_ptr(), spec2.data_ptr(), nx, ny, nz, tables.data_ptr(), masks, gk,
         ptr(transfer), ptr(radial), rl, post, s)
    call("pmb_interlace_spectra", spec2.data_ptr(), spec2.data_ptr() + 8 * Mc, nx, ny, nz, 1, s)
    t = timer.mark("green_gradient", t)
    call("pmb_irfft3", nx, ny, nz, 2, spec2.data_ptr(), real3.data_ptr(), work.data_ptr(), s)
    t = timer.mark("fft_c2r", t)
    vc = float(conf.mesh_size / conf.ptcl_num)
    for k, sb in enumerate((sorted_buf, sorted_sh)):
        call("pmb_interp_grad_rows", sb.data_ptr(), n, nx, ny, nz, 1, real3.data_ptr() + 4 * M * k, None, vc,
             float(conf.cell_size), 1, disp_cot.data_ptr(), None, None, s)
    timer.mark("scatter_adjoint", t)


class _NoTimer:
    def start(self):
        return None

    def mark(self, name, start):
        return None

    def tag(self, name):
        return None


def _force_staged(pmid, disp, conf, omega_m, tables, gk, transfer, radial, rl, F, acc, drift_vel, drift, vel_kick,
                  kick, timer, src_hat_out=None, lane="", kick2=0.0, keep_acc=True):
    """pmb_force as separate stage calls with a CUDA event after each stage.

    With src_hat_out (complex64, half spectrum) the rFFT of the Poisson source
    is kept there (the learned correction's adjoint needs it)."""
    n = pmid.shape[0]
    nx, ny, nz = conf.mesh_shape
    dev = disp.device
    s = stream_handle(dev)
    sorted_buf, sort_scr, s16, real3 = _stage_buffers(n, conf, dev, sorted_lane=lane)
    timer = _NoTimer() if timer is None else timer
    t = timer.start()
    call("pmb_sort_rows", pmid.data_ptr(), disp.data_ptr(), ptr(drift_vel), float(drift), n, nx, ny, nz,
         float(conf.cell_size), sorted_buf.data_ptr(), sort_scr.data_ptr(), sort_scr.numel(), s)
    t = timer.mark("sort", t)
    call("pmb_scatter_rows", sorted_buf.data_ptr(), n, nx, ny, nz, 1, None, 0, float(conf.mesh_size / conf.ptcl_num),
         1, 1.5 * _om32(omega_m), real3.data_ptr(), s16.data_ptr(), s)
    t = timer.mark("scatter", t)
    masks = int(conf.has_particle_nyquist_masks)
    if src_hat_out is None and pmfft_active(nx, ny, nz):
        # hand-written pass chain (pmfft.cu): z R2C, y, x + Green + x^-1, y^-1, z C2R
        C8 = 8 * lib().pmb_pmfft_channel_elems(nx, ny, nz)
        pm = workspace(5 * C8, dev, "st_pm5")
        aq, fp = pm.data_ptr(), pm.data_ptr() + 2 * C8
        # (pruned to the live spectrum when the particle-Nyquist masks apply)
        tp = tables.data_ptr()
        call("pmb_pmfft_z2", nx, ny, nz, 0, 1, real3.data_ptr(), aq, tp, masks, masks, s)
        t = timer.mark("fft_z_r2c", t)
        call("pmb_pmfft_col2", nx, ny, nz, 0, 1, 0, aq, fp, tp, masks, None, None, 0, 1.0, masks, s)
        t = timer.mark("fft_y", t)
        call("pmb_pmfft_col2", nx, ny, nz, 6, 1, 0, fp, aq, tp, masks, ptr(transfer), ptr(radial), rl,
             float(1.0 / conf.mesh_size), masks, s)
        t = timer.mark("fft_x_green", t)
        call("pmb_pmfft_col2", nx, ny, nz, 1, 1, 0, aq, fp, tp, masks, None, None, 0, 1.0, masks, s)
        t = timer.mark("fft_y_inv", t)
        call("pmb_pmfft_col2", nx, ny, nz, 2, 1, 1, aq, fp + C8, tp, masks, None, None, 0, 1.0, masks, s)
        t = timer.mark("fft_y_inv_yz", t)
        call("pmb_pmfft_z2", nx, ny, nz, 1, 3, fp, F.data_ptr(), tp, masks, masks, s)
        t = timer.mark("fft_z_c2r3", t)
    else:
        spec3, spec1, work = _cufft_buffers(conf, dev)
        if src_hat_out is not None:
            spec1 = src_hat_out
        call("pmb_rfft3", nx, ny, nz, 1, real3.data_ptr(), spec1.data_ptr(), work.data_ptr(), s)
        t = timer.mark("fft_r2c", t)
        call("pmb_green_gradient", spec1.data_ptr(), spec3.data_ptr(), nx, ny, nz, tables.data_ptr(), masks, gk,
             ptr(transfer), ptr(radial), rl, float(1.0 / conf.mesh_size), s)
        t = timer.mark("green_gradient", t)
        call("pmb_irfft3", nx, ny, nz, 3, spec3.data_ptr(), F.data_ptr(), work.data_ptr(), s)
        t = timer.mark("fft_c2r", t)
    out = acc if (keep_acc or vel_kick is None) else None
    call("pmb_gather_rows2", sorted_buf.data_ptr(), n, nx, ny, nz, 3, F.data_ptr(), ptr(out), ptr(vel_kick),
         float(kick), float(kick2), s)
    timer.mark("gather", t)
    if vel_kick is not None:
        # this gather also read and wrote the velocities (and stored no acc)
        timer.tag("gather_kick" if out is not None else "gather_kick_only")


def _force_vjp_staged(pmid, disp, conf, omega_m, tables, gk, transfer, radial, rl, F, acc_cot, disp_cot, timer,
                      src_hat=None, transfer_cot_out=None, presorted=False, sorted_lane="", work_lane=""):
    """pmb_force_vjp as separate stage calls with a CUDA event after each stage.

    With src_hat (the source spectrum at the same positions) and
    transfer_cot_out (float64, radial table length) also accumulates dL/dT per
    integer |n|^2 (pmb_transfer_cot)."""
    n = pmid.shape[0]
    nx, ny, nz = conf.mesh_shape
    dev = disp.device
    s = stream_handle(dev)
    sorted_buf, sort_scr, s16, real3 = _stage_buffers(n, conf, dev, sorted_lane if presorted else work_lane,
                                                      work_lane)
    timer = _NoTimer() if timer is None else timer
    t = timer.start()
    if not presorted:
        call("pmb_sort_rows", pmid.data_ptr(), disp.data_ptr(), None, 0.0, n, nx, ny, nz, float(conf.cell_size),
             sorted_buf.data_ptr(), sort_scr.data_ptr(), sort_scr.numel(), s)
        t = timer.mark("sort", t)
    cot_sorted = workspace(12 * n, dev, "st_cot_sorted" + work_lane)
    call("pmb_interp_grad_rows", sorted_buf.data_ptr(), n, nx, ny, nz, 3, F.data_ptr(), acc_cot.data_ptr(), 0.0,
         float(conf.cell_size), 1, disp_cot.data_ptr(), None, cot_sorted.data_ptr(), s)
    t = timer.mark("gather_adjoint", t)
    call("pmb_scatter_rows", sorted_buf.data_ptr(), n, nx, ny, nz, 3, cot_sorted.data_ptr(), 1, 0.0, 0, 1.0,
         real3.data_ptr(), s16.data_ptr(), s)
    t = timer.mark("scatter3", t)
    post = float(np.float32(1.5 * _om32(omega_m)) / conf.mesh_size)
    masks = int(conf.has_particle_nyquist_masks)
    if transfer_cot_out is None and pmfft_active(nx, ny, nz):
        # transposed pass chain: z R2C x3, y (x channel; y and z folded), x + adjoint multiplier + x^-1, y^-1, z C2R
        C8 = 8 * lib().pmb_pmfft_channel_elems(nx, ny, nz)
        pm = workspace(5 * C8, dev, "st_pm5" + work_lane)
        a3, bb = pm.data_ptr(), pm.data_ptr() + 3 * C8
        tp = tables.data_ptr()
        call("pmb_pmfft_z2", nx, ny, nz, 0, 3, real3.data_ptr(), a3, tp, masks, masks, s)
        t = timer.mark("fft_z_r2c3", t)
        call("pmb_pmfft_col2", nx, ny, nz, 0, 1, 0, a3, bb, tp, masks, None, None, 0, 1.0, masks, s)
        t = timer.mark("fft_y", t)
        call("pmb_pmfft_col2", nx, ny, nz, 3, 1, 1, a3, bb + C8, tp, masks, None, None, 0, 1.0, masks, s)
        t = timer.mark("fft_y_yz", t)
        call("pmb_pmfft_col2", nx, ny, nz, 7, 1, 0, bb, a3, tp, masks, ptr(transfer), ptr(radial), rl, post, masks, s)
        t = timer.mark("fft_x_green_adj", t)
        call("pmb_pmfft_col2", nx, ny, nz, 1, 1, 0, a3, a3 + C8, tp, masks, None, None, 0, 1.0, masks, s)
        t = timer.mark("fft_y_inv", t)
        call("pmb_pmfft_z2", nx, ny, nz, 1, 1, a3 + C8, real3.data_ptr(), tp, masks, masks, s)
        t = timer.mark("fft_z_c2r", t)
    else:
        spec3, spec1, work = _cufft_buffers(conf, dev)
        call("pmb_rfft3", nx, ny, nz, 3, real3.data_ptr(), spec3.data_ptr(), work.data_ptr(), s)
        t = timer.mark("fft_r2c", t)
        if transfer_cot_out is not None:
            call("pmb_transfer_cot", spec3.data_ptr(), src_hat.data_ptr(), nx, ny, nz, tables.data_ptr(), masks,
                 int(transfer_cot_out.numel()), transfer_cot_out.data_ptr(), s)
        call("pmb_green_gradient_adjoint", spec3.data_ptr(), spec1.data_ptr(), nx, ny, nz, tables.data_ptr(), masks,
             gk, ptr(transfer), ptr(radial), rl, post, s)
        t = timer.mark("green_gradient", t)
        call("pmb_irfft3", nx, ny, nz, 1, spec1.data_ptr(), real3.data_ptr(), work.data_ptr(), s)
        t = timer.mark("fft_c2r", t)
    call("pmb_interp_grad_rows", sorted_buf.data_ptr(), n, nx, ny, nz, 1, real3.data_ptr(), None,
         float(conf.mesh_size / conf.ptcl_num), float(conf.cell_size), 1, disp_cot.data_ptr(), None, None, s)
    timer.mark("scatter_adjoint", t)


def _correction_args(correction, a, cosmo, conf):
    if correction is None:
        return 0, None, None, 0
    gk = int(getattr(correction, "green_kernel", 0))
    transfer, radial = correction.transfer_tables(a, cosmo, conf)
    rl = 0 if radial is None else int(radial.numel())
    return gk, transfer, radial, rl


def _tables(conf, dev, gk, correction):
    """Spectral tables for the correction's Green's function and force
    derivative (corrections/core.py:396-422: force_green_kernel,
    force_gradient_kernel)."""
    grad = getattr(correction, "gradient_kernel", "spectral") if correction is not None else "spectral"
    if grad not in ("spectral", "fastpm_4point"):
        raise ValueError(f"Unsupported force-gradient kernel {grad!r}.")
    return conf.spectral_tables("mesh", dev, gk, 1 if grad == "fastpm_4point" else 0)


def force(pmid, disp, conf, omega_m, *, a=None, cosmo=None, correction=None, force_meshes=None, acc=None,
          drift_vel=None, drift=0.0, vel_kick=None, kick=0.0, kick2=0.0, src_hat_out=None, lane="", keep_acc=True):
    """One PM force evaluation on device tensors.

    Returns (acc (N,3), force_meshes (3,Mx,My,Mz)).  With drift_vel the
    particles are drifted first (disp updated in place); with vel_kick the
    half-kick vel_kick += acc * kick is fused into the gather, followed by
    vel_kick += acc * kick2 when kick2 != 0 (the next step's opening kick).
    lane selects the workspace that keeps the sorted records (see force_vjp).
    keep_acc=False with vel_kick: apply the kicks without storing acc (the
    plain route; returns acc None there).
    float64 displacements take the float64 build (x64.force: the analytic
    corrections, one folded kick)."""
    require_cuda(pmid, disp, drift_vel, vel_kick)
    if disp.dtype == torch.float64:
        if kick2 != 0.0 or src_hat_out is not None:
            raise NotImplementedError("the float64 force takes one folded kick and no spectrum")
        from . import x64
        return x64.force(pmid, disp, conf, omega_m, acc=acc, force_meshes=force_meshes, drift_vel=drift_vel,
                         drift=drift, vel_kick=vel_kick, kick=kick, correction=correction, a=a, cosmo=cosmo)
    n = pmid.shape[0]
    nx, ny, nz = conf.mesh_shape
    dev = disp.device
    if force_meshes is None:
        force_meshes = torch.empty((3, nx, ny, nz), dtype=torch.float32, device=dev)
    if acc is None:
        acc = torch.empty((n, 3), dtype=torch.float32, device=dev)
    gk, transfer, radial, rl = _correction_args(correction, a, cosmo, conf)
    tables = _tables(conf, dev, gk, correction)
    cnn = mesh_cnn_of(correction)
    if cnn is not None:
        if uses_interlacing(correction) or src_hat_out is not None:
            raise NotImplementedError("the mesh-CNN correction takes no interlacing and no learned radial transfer")
        _force_cnn(pmid, disp, conf, omega_m, tables, gk, transfer, radial, rl, force_meshes, acc, drift_vel, drift,
                   vel_kick, kick, kick2, StageTimer.active, cnn, a, cosmo, lane)
        return acc, force_meshes
    if uses_interlacing(correction):
        _force_interlaced(pmid, disp, conf, omega_m, tables, gk, transfer, radial, rl, force_meshes, acc, drift_vel,
                          drift, vel_kick, kick, kick2, StageTimer.active, src_hat_out, lane)
        return acc, force_meshes
    if StageTimer.active is not None or src_hat_out is not None:
        _force_staged(pmid, disp, conf, omega_m, tables, gk, transfer, radial, rl, force_meshes, acc, drift_vel,
                      drift, vel_kick, kick, StageTimer.active, src_hat_out, lane, kick2, keep_acc)
        return (acc if (keep_acc or vel_kick is None) else None), force_meshes
    wb = lib().pmb_force_workspace_bytes(n, nx, ny, nz)
    if wb < 0:
        raise RuntimeError("pmb_force_workspace_bytes failed: " + lib().pmb_last_error().decode())
    ws = workspace(wb, dev, "force" + _lane_suffix(lane))
    out = acc if (keep_acc or vel_kick is None) else None
    call("pmb_force2", pmid.data_ptr(), disp.data_ptr(), ptr(drift_vel), float(drift), n, nx, ny, nz,
         float(conf.cell_size), float(conf.mesh_size / conf.ptcl_num), 1.5 * _om32(omega_m), tables.data_ptr(),
         int(conf.has_particle_nyquist_masks), gk, ptr(transfer), ptr(radial), rl, force_meshes.data_ptr(),
         ptr(out), ptr(vel_kick), float(kick), float(kick2), ws.data_ptr(), ws.numel(), stream_handle(dev))
    return out, force_meshes


def force_vjp(pmid, disp, conf, omega_m, force_meshes, acc_cot, disp_cot=None, *, a=None, cosmo=None,
              correction=None, src_hat=None, transfer_cot_out=None, presorted=False, sorted_lane="",
              concurrent=False, om_out=None):
    """disp_cot (+)= (d acc / d disp)^T acc_cot, with force_meshes computed at disp.

    presorted: the last force() call with lane=sorted_lane was at exactly
    these positions and took the same route (fused or staged); its
    cell-sorted records are reused instead of sorting again (disp is then not
    read).  concurrent: use workspaces of its own so that a force() may run on
    another stream at the same time.  float64 displacements take
    x64.force_vjp.  om_out (a list) receives the force's Omega_m cotangent
    where it is not sum(acc_cot acc) / Omega_m (the mesh-CNN correction)."""
    require_cuda(pmid, disp, force_meshes, acc_cot, disp_cot)
    if disp.dtype == torch.float64:
        if transfer_cot_out is not None or src_hat is not None:
            raise NotImplementedError("the float64 force adjoint trains no correction")
        from . import x64
        return x64.force_vjp(pmid, disp, conf, omega_m, force_meshes, acc_cot, disp_cot, correction=correction, a=a,
                             cosmo=cosmo)
    n = pmid.shape[0]
    nx, ny, nz = conf.mesh_shape
    dev = disp.device
    if disp_cot is None:
        disp_cot = torch.zeros((n, 3), dtype=torch.float32, device=dev)
    gk, transfer, radial, rl = _correction_args(correction, a, cosmo, conf)
    tables = _tables(conf, dev, gk, correction)
    cnn = mesh_cnn_of(correction)
    if cnn is not None:
        if uses_interlacing(correction) or transfer_cot_out is not None:
            raise NotImplementedError("the mesh-CNN correction takes no interlacing and no learned radial transfer")
        _force_vjp_cnn(pmid, disp, conf, omega_m, tables, gk, transfer, radial, rl, force_meshes, acc_cot, disp_cot,
                       StageTimer.active, cnn, a, cosmo, presorted, sorted_lane, "v" if concurrent else "", om_out)
        return disp_cot
    if uses_interlacing(correction):
        _force_vjp_interlaced(pmid, disp, conf, omega_m, tables, gk, transfer, radial, rl, force_meshes, acc_cot,
                              disp_cot, StageTimer.active, src_hat, transfer_cot_out, presorted, sorted_lane,
                              "v" if concurrent else "")
        return disp_cot
    if StageTimer.active is not None or transfer_cot_out is not None:
        _force_vjp_staged(pmid, disp, conf, omega_m, tables, gk, transfer, radial, rl, force_meshes, acc_cot,
                          disp_cot, StageTimer.active, src_hat, transfer_cot_out, presorted, sorted_lane,
                          "v" if concurrent else "")
        return disp_cot
    wb = lib().pmb_force_vjp_workspace_bytes(n, nx, ny, nz)
    ws = workspace(wb, dev, "force_vjp")
    if presorted:
        # head of the fused force's workspace: its sorted records
        head = workspace(lib().pmb_force_workspace_bytes(n, nx, ny, nz), dev, "force" + _lane_suffix(sorted_lane))
        call("pmb_force_vjp_presorted", head.data_ptr(), n, nx, ny, nz, float(conf.cell_size),
             float(conf.mesh_size / conf.ptcl_num), 1.5 * _om32(omega_m), tables.data_ptr(),
             int(conf.has_particle_nyquist_masks), gk, ptr(transfer), ptr(radial), rl, force_meshes.data_ptr(),
             acc_cot.data_ptr(), disp_cot.data_ptr(), ws.data_ptr(), ws.numel(), stream_handle(dev))
        return disp_cot
    call("pmb_force_vjp", pmid.data_ptr(), disp.data_ptr(), n, nx, ny, nz, float(conf.cell_size),
         float(conf.mesh_size / conf.ptcl_num), 1.5 * _om32(omega_m), tables.data_ptr(),
         int(conf.has_particle_nyquist_masks), gk, ptr(transfer), ptr(radial), rl, force_meshes.data_ptr(),
         acc_cot.data_ptr(), disp_cot.data_ptr(), ws.data_ptr(), ws.numel(), stream_handle(dev))
    return disp_cot


def force_streamed(pmid, disp, conf, omega_m, *, acc=None, drift_vel=None, drift=0.0):
    """The low-memory forward force (pmb_force_streamed): one force component
    at a time through one real mesh; forward only."""
    require_cuda(pmid, disp, drift_vel)
    n = pmid.shape[0]
    nx, ny, nz = conf.mesh_shape
    dev = disp.device
    if acc is None:
        acc = torch.empty((n, 3), dtype=torch.float32, device=dev)
    wb = lib().pmb_force_streamed_workspace_bytes(n, nx, ny, nz)
    if wb < 0:
        raise RuntimeError("pmb_force_streamed_workspace_bytes failed: " + lib().pmb_last_error().decode())
    ws = workspace(wb, dev, "force_streamed")
    tables = conf.spectral_tables("mesh", dev, 0)
    call("pmb_force_streamed", pmid.data_ptr(), disp.data_ptr(), ptr(drift_vel), float(drift), n, nx, ny, nz,
         float(conf.cell_size), float(conf.mesh_size / conf.ptcl_num), 1.5 * _om32(omega_m), tables.data_ptr(),
         int(conf.has_particle_nyquist_masks), 0, None, None, 0, acc.data_ptr(), ws.data_ptr(), ws.numel(),
         stream_handle(dev))
    return acc


def gravity_streamed(a, ptcl, cosmo, conf, correction=None):
    """Uncorrected PM accelerations with sequential component FFTs
    (nbody/gravity.py:643-658): the memory-lean forward path."""
    if correction is not None:
        raise ValueError("streamed gravity currently requires correction=None.")
    return force_streamed(ptcl.pmid, ptcl.disp, conf, cosmo.Omega_m)


def gravity(a, ptcl, cosmo, conf, correction=None):
    """Gravitational accelerations [H_0^2 L] (gravity.py:786-814)."""
    acc, _ = force(ptcl.pmid, ptcl.disp, conf, cosmo.Omega_m, a=a, cosmo=cosmo, correction=correction)
    return acc


def gravity_vjp(a, ptcl, cosmo, conf, acc_cot, correction=None):
    """Returns (disp_cot, Omega_m_cot) of gravity w.r.t. acc_cot."""
    acc, F = force(ptcl.pmid, ptcl.disp.clone(), conf, cosmo.Omega_m, a=a, cosmo=cosmo, correction=correction)
    om_out = []
    dc = force_vjp(ptcl.pmid, ptcl.disp, conf, cosmo.Omega_m, F, acc_cot.contiguous(), a=a, cosmo=cosmo,
                   correction=correction, om_out=om_out)
    if om_out:
        return dc, om_out[0]
    om = float(cosmo.Omega_m) if acc.dtype == torch.float64 else _om32(cosmo.Omega_m)
    om_cot = float((acc_cot.double() * acc.double()).sum()) / om
    return dc, om_cot
