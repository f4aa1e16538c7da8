"""Lagrangian perturbation theory initial conditions (initial_conditions/lpt.py:337-449).

``lpt(modes, cosmo, conf)`` builds 1LPT/2LPT displacements and canonical
velocities on the Lagrangian lattice at conf.a_start from linear modes on the
particle grid, entirely through the fused C-ABI call pmb_lpt (strain spectra,
one batched C2R, the quadratic 2LPT source, R2C, six gradient C2Rs,
sampling).  ``lpt_vjp`` is the hand-written adjoint w.r.t. the modes and the
growth factors.
"""
from __future__ import annotations

import numpy as np
import torch

from ._lib import call, lib
from .particles import Particles
from .runtime import ptr, stream_handle, workspace


class LPTResult:
    """Particles plus what the adjoint needs (sampled gradient fields, grid index)."""

    def __init__(self, ptcl, modes, fields, index, factors, dfactors):
        self.ptcl = ptcl
        self.modes = modes
        self.fields = fields
        self.index = index
        self.factors = factors
        self.dfactors = dfactors


def lpt_full(modes, cosmo, conf):
    if conf.float_dtype == torch.float64:
        from . import x64
        return x64.lpt_full(modes, cosmo, conf)
    gx, gy, gz = conf.ptcl_grid_shape
    dev = modes.device
    modes = modes.contiguous()
    ptcl = Particles.gen_grid(conf, vel=True, device=dev)
    fac, dfac = cosmo.lpt_factors(conf.a_start)
    f32 = lambda x: float(np.float32(x))
    D1, V1, D2, V2 = f32(fac[0, 0]), f32(fac[0, 2]), f32(fac[1, 0]), f32(fac[1, 2])
    fields = torch.empty((6, gx, gy, gz), dtype=torch.float32, device=dev)
    index = torch.empty(len(ptcl), dtype=torch.int64, device=dev)
    tables = conf.spectral_tables("particle", dev)
    ws = workspace(lib().pmb_lpt_workspace_bytes(gx, gy, gz), dev, "lpt")
    call("pmb_lpt", modes.data_ptr(), gx, gy, gz, float(conf.ptcl_spacing), float(conf.ptcl_cell_vol),
         tables.data_ptr(), int(conf.lpt_order), D1, V1, D2, V2, ptcl.pmid.data_ptr(), ptcl.disp.data_ptr(),
         ptcl.vel.data_ptr(), len(ptcl), float(conf.cell_size), fields.data_ptr(), index.data_ptr(), ws.data_ptr(),
         ws.numel(), stream_handle(dev))
    return LPTResult(ptcl, modes, fields, index, fac, dfac)


def lpt(modes, cosmo, conf):
    """LPT particles at conf.a_start (acc unset)."""
    if conf.float_dtype == torch.float64:
        from . import x64
        return x64.lpt(modes, cosmo, conf)
    return lpt_full(modes, cosmo, conf).ptcl


def lpt_vjp(res, disp_cot, vel_cot, cosmo, conf, amp=None):
    """Adjoint of lpt: returns (modes_cot, Omega_m_cot from the growth factors).

    modes_cot uses the packed convention dL/dRe + i dL/dIm per stored rFFT
    coefficient (the complex conjugate of JAX's gradient of a real loss).  With
    amp the cotangent is chained through the linear-mode amplitude (the result
    is then w.r.t. the white-noise modes)."""
    if res.modes.dtype == torch.complex128:
        from . import x64
        return x64.lpt_vjp(res, disp_cot, vel_cot, cosmo, conf, amp)
    gx, gy, gz = conf.ptcl_grid_shape
    dev = res.modes.device
    order = int(conf.lpt_order)
    f32 = lambda x: float(np.float32(x))
    fac = res.factors
    mc = torch.empty_like(res.modes)
    if order == 0:
        mc.zero_()
        return mc, 0.0
    dots = torch.zeros(4, dtype=torch.float64, device=dev)
    ws = workspace(lib().pmb_lpt_vjp_workspace_bytes(gx, gy, gz), dev, "lpt_vjp")
    call("pmb_lpt_vjp", res.modes.data_ptr(), gx, gy, gz, float(conf.ptcl_cell_vol),
         conf.spectral_tables("particle", dev).data_ptr(), order, f32(fac[0, 0]), f32(fac[0, 2]), f32(fac[1, 0]),
         f32(fac[1, 2]), res.index.data_ptr(), res.fields.data_ptr(), disp_cot.contiguous().data_ptr(),
         vel_cot.contiguous().data_ptr(), res.index.numel(), ptr(amp), mc.data_ptr(), dots.data_ptr(), ws.data_ptr(),
         ws.numel(), stream_handle(dev))
    d = dots.cpu().numpy()
    dfac = res.dfactors
    om = 0.0
    for m in range(order):
        om += dfac[m, 0] * d[2 * m] + dfac[m, 2] * d[2 * m + 1]
    return mc, float(om)
