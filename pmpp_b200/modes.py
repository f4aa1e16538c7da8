"""White-noise and linear-mode initial conditions on the device.

Mirrors initial_conditions/modes.py: ``white_noise_nested(seed, conf)``
(:223-268, resolution-consistent hashed Gaussian modes) and
``linear_modes(modes, cosmo, conf, a=None)`` (:397-454,
delta(k) = omega(k) sqrt(V P_lin(k))).  Fourier modes are complex64 tensors of
shape (gx, gy, gz//2 + 1) in the rFFT layout.
"""
from __future__ import annotations

import numpy as np
import torch

from ._lib import call, lib
from .cosmology import growth, transfer_fit
from .runtime import ptr, stream_handle, workspace


def _grid(conf):
    return conf.ptcl_grid_shape


def white_noise_nested(seed, conf, real=False, unit_abs=False, device=None, return_hashes=False):
    """Hashed Gaussian rFFT modes (modes.py:181-268); complex128 in the float64 build."""
    device = conf.device if device is None else torch.device(device)
    if conf.float_dtype == torch.float64:
        if real or unit_abs or return_hashes:
            raise NotImplementedError("the float64 build returns the complex modes only")
        from . import x64
        return x64.white_noise_nested(seed, conf, device)
    gx, gy, gz = _grid(conf)
    out = torch.empty((gx, gy, gz // 2 + 1), dtype=torch.complex64, device=device)
    hashes = torch.empty((gx, gy, gz // 2 + 1, 2), dtype=torch.int32, device=device) if return_hashes else None
    call("pmb_white_noise_nested", int(seed) & 0xFFFFFFFF, gx, gy, gz, out.data_ptr(), ptr(hashes),
         stream_handle(device))
    if unit_abs:
        norm = out.abs()
        out = torch.where(norm != 0, out / norm, torch.ones_like(out))
    if real:
        out = irfft3(out, conf.ptcl_grid_shape) / np.sqrt(conf.ptcl_num)
    return (out, hashes) if return_hashes else out


def irfft3(spec, shape):
    """Unnormalised C2R (cuFFT through the C ABI); the input is not modified."""
    nx, ny, nz = shape
    dev = spec.device
    src = spec.contiguous().clone()
    out = torch.empty(shape, dtype=torch.float32, device=dev)
    w = workspace(lib().pmb_fft_work_bytes(nx, ny, nz, 1), dev, "fft1")
    call("pmb_irfft3", nx, ny, nz, 1, src.data_ptr(), out.data_ptr(), w.data_ptr(), stream_handle(dev))
    return out


def rfft3(x):
    nx, ny, nz = x.shape
    dev = x.device
    out = torch.empty((nx, ny, nz // 2 + 1), dtype=torch.complex64, device=dev)
    w = workspace(lib().pmb_fft_work_bytes(nx, ny, nz, 1), dev, "fft1")
    xin = x.contiguous().to(torch.float32)
    call("pmb_rfft3", nx, ny, nz, 1, xin.data_ptr(), out.data_ptr(), w.data_ptr(), stream_handle(dev))
    return out


class _Tables:
    def __init__(self, cosmo, conf, device):
        self.tk = torch.from_numpy(np.ascontiguousarray(conf.transfer_k, dtype=np.float64)).to(device)
        self.tt = torch.from_numpy(np.ascontiguousarray(cosmo.transfer, dtype=np.float64)).to(device)
        self.k = torch.from_numpy(np.concatenate(conf.kvec_spacing).astype(np.float32)).to(device)


def _linear_call(modes_in, modes_out, amp_out, cosmo, conf, a, transfer=None, omega_m=None, A_s=None):
    device = (modes_out if modes_out is not None else amp_out).device
    gx, gy, gz = _grid(conf)
    tb = _Tables(cosmo, conf, device)
    tt = tb.tt if transfer is None else torch.from_numpy(np.ascontiguousarray(transfer, dtype=np.float64)).to(device)
    g2 = 1.0 if a is None else float(growth(float(np.float32(a)), cosmo, conf))**2
    call("pmb_linear_modes", ptr(modes_in), ptr(modes_out), ptr(amp_out), gx, gy, gz, tb.k.data_ptr(),
         tb.tk.data_ptr(), tt.data_ptr(), int(tb.tk.numel()), float(cosmo.A_s if A_s is None else A_s),
         float(cosmo.n_s), float(cosmo.Omega_m if omega_m is None else omega_m), float(cosmo.k_pivot), g2,
         float(conf.box_vol), stream_handle(device))


def linear_modes(modes, cosmo, conf, a=None, real=False):
    """delta(k) = omega(k) sqrt(V P_lin(|k|, a)) (modes.py:397-454)."""
    if conf.float_dtype == torch.float64:
        if a is not None or real or not torch.is_complex(modes):
            raise NotImplementedError("the float64 build takes complex modes at a = 1")
        from . import x64
        return x64.linear_modes(modes, cosmo, conf)
    if not torch.is_complex(modes):
        modes = rfft3(modes) / np.sqrt(conf.ptcl_num)
    modes = modes.contiguous()
    out = torch.empty_like(modes)
    _linear_call(modes, out, None, cosmo, conf, a)
    if real:
        return irfft3(out, conf.ptcl_grid_shape) / conf.ptcl_num
    return out


def linear_amplitude(cosmo, conf, a=None, device=None):
    """sqrt(V P_lin(|k|)) per rFFT cell (float32; float64 in the float64 build, at a = 1)."""
    device = conf.device if device is None else torch.device(device)
    if conf.float_dtype == torch.float64:
        if a is not None:
            raise NotImplementedError("the float64 build takes the linear amplitude at a = 1")
        from . import x64
        return x64.linear_amplitude(cosmo, conf, device)
    gx, gy, gz = _grid(conf)
    amp = torch.empty((gx, gy, gz // 2 + 1), dtype=torch.float32, device=device)
    _linear_call(None, None, amp, cosmo, conf, a)
    return amp


def linear_modes_param_cotangents(omega, modes_cot, cosmo, conf, a=None, h=1e-6):
    """(dL/dA_s_1e9, dL/dOmega_m) of the linear modes given their cotangent.

    A_s enters as sqrt(A_s) (exact); Omega_m through the transfer function and
    the explicit 1/Omega_m: the modes are re-evaluated with the transfer table
    differentiated in FP64 (central difference of the analytic fit)."""
    if conf.float_dtype == torch.float64:
        if a is not None:
            raise NotImplementedError("the float64 build takes the linear modes at a = 1")
        from . import x64
        return x64.linear_modes_param_cotangents(omega, modes_cot, cosmo, conf, h=h)
    dev = omega.device
    s = stream_handle(dev)
    lin = torch.empty_like(omega)
    _linear_call(omega, lin, None, cosmo, conf, a)
    dots = torch.zeros(4, dtype=torch.float64, device=dev)
    n2 = 2 * omega.numel()
    mc = torch.view_as_real(modes_cot.contiguous())
    call("pmb_dot", mc.data_ptr(), torch.view_as_real(lin).data_ptr(), n2, dots[0:].data_ptr(), s)
    # Omega_m: P ~ (T / Omega_m)^2, so dA/dOm = A (dT/dOm / T - 1/Om); evaluate
    # the two pieces with the kernel at transfer tables (T +- h dT) and Om.
    Tp = transfer_fit(conf.transfer_k, cosmo.replace(Omega_m=cosmo.Omega_m + h), conf)
    Tm = transfer_fit(conf.transfer_k, cosmo.replace(Omega_m=cosmo.Omega_m - h), conf)
    dT = (Tp - Tm) / (2 * h)
    eps = 1e-2
    while np.any(cosmo.transfer[1:] - eps * np.abs(dT[1:]) <= 0):
        eps *= 0.5
    up = torch.empty_like(omega)
    dn = torch.empty_like(omega)
    _linear_call(omega, up, None, cosmo, conf, a, transfer=cosmo.transfer + eps * dT)
    _linear_call(omega, dn, None, cosmo, conf, a, transfer=cosmo.transfer - eps * dT)
    call("pmb_dot", mc.data_ptr(), torch.view_as_real(up).data_ptr(), n2, dots[1:].data_ptr(), s)
    call("pmb_dot", mc.data_ptr(), torch.view_as_real(dn).data_ptr(), n2, dots[2:].data_ptr(), s)
    d = dots.cpu().numpy()
    dA_s_1e9 = d[0] / (2 * cosmo.A_s_1e9)
    # A is linear in T, so the central difference in T is exact up to rounding
    dOm = (d[1] - d[2]) / (2 * eps) - d[0] / cosmo.Omega_m
    return float(dA_s_1e9), float(dOm)
