"""Isotropic power spectrum with FP64 shell sums (analysis/power_spectrum.py).

``delta_to_pk``, ``density_to_pk``, ``particles_to_pk`` and the
cross-correlation variants return (k, P(k), nmodes) over integer-radius shells
1..n-1 with the CIC window deconvolution and the rFFT multiplicity of the
reference (:46-143, :251-305).  ``log_binned`` rebins shells into log-spaced
bins weighted by mode count (an extension for the 32-log-bin outputs; the
reference reports integer shells only).  ``pk_loss`` is the mean squared log
ratio against a target spectrum with its hand-written gradient back to
particle displacements.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from ._lib import call, lib
from .cic import SortedParticles
from .runtime import stream_handle, workspace

_MAS_POWER = {None: 0, "NGP": 1, "CIC": 2, "TSC": 3, "PCS": 4}
_stats_cache = {}


def _mas(mas):
    if mas is None:
        return 0
    m = mas.upper()
    if m not in _MAS_POWER:
        raise ValueError(f"Unsupported MAS={mas!r}")
    return _MAS_POWER[m]


def num_shells(conf):
    return math.floor(math.sqrt(3) * (conf.mesh_shape[0] // 2)) + 1


def _sinc_tables(conf, device):
    key = ("sinc", conf.mesh_shape, str(device))
    if key not in _stats_cache:
        nx, ny, nz = conf.mesh_shape
        parts = []
        for n, modes in ((nx, np.fft.fftfreq(nx) * nx), (ny, np.fft.fftfreq(ny) * ny), (nz, np.arange(nz // 2 + 1))):
            x = (modes.astype(np.float32) / np.float32(n)).astype(np.float32)
            parts.append(np.sinc(x.astype(np.float64)).astype(np.float32))
        _stats_cache[key] = torch.from_numpy(np.concatenate(parts)).to(device)
    return _stats_cache[key]


def shell_statistics(conf, device=None):
    """(k centres float64 numpy, nmodes int64 numpy) over shells >= 1 (:46-74)."""
    device = conf.device if device is None else torch.device(device)
    key = ("stats", conf.mesh_shape, conf.cell_size, str(device))
    if key not in _stats_cache:
        nx, ny, nz = conf.mesh_shape
        ns = num_shells(conf) + 1  # statistics may reach one shell further
        counts = torch.empty(ns, dtype=torch.float64, device=device)
        ksum = torch.empty(ns, dtype=torch.float64, device=device)
        call("pmb_shell_stats", nx, ny, nz, ns, counts.data_ptr(), ksum.data_ptr(), stream_handle(device))
        c = counts.cpu().numpy()
        kk = ksum.cpu().numpy() / np.maximum(c, 1) * (2 * math.pi / (nx * conf.cell_size))
        _stats_cache[key] = (kk[1:], c[1:].astype(np.int64))
    return _stats_cache[key]


def _spectrum(delta, conf):
    nx, ny, nz = conf.mesh_shape
    dev = delta.device
    x = delta.to(torch.float32).contiguous()
    spec = torch.empty((nx, ny, nz // 2 + 1), dtype=torch.complex64, device=dev)
    w = workspace(lib().pmb_fft_work_bytes(nx, ny, nz, 1), dev, "fft1")
    call("pmb_rfft3", nx, ny, nz, 1, x.data_ptr(), spec.data_ptr(), w.data_ptr(), stream_handle(dev))
    return spec


def _shell_sums(spec, conf, mas_power, spec_b=None):
    nx, ny, nz = conf.mesh_shape
    dev = spec.device
    ns = num_shells(conf)
    sums = torch.empty(ns, dtype=torch.float64, device=dev)
    sb = torch.empty(ns, dtype=torch.float64, device=dev) if spec_b is not None else None
    sx = torch.empty(ns, dtype=torch.float64, device=dev) if spec_b is not None else None
    call("pmb_pk_shells", spec.data_ptr(), nx, ny, nz, _sinc_tables(conf, dev).data_ptr(), mas_power, ns,
         sums.data_ptr(), None if spec_b is None else spec_b.data_ptr(), None if sb is None else sb.data_ptr(),
         None if sx is None else sx.data_ptr(), stream_handle(dev))
    return sums, sb, sx


def _finalize(p_sum, conf):
    """:251-256: P = sum[1:] / nmodes * cell^3 / M."""
    k, nmodes = shell_statistics(conf)
    ns = num_shells(conf) - 1
    k, nmodes = k[:ns], nmodes[:ns]
    pk = p_sum.cpu().numpy()[1:] / nmodes * (conf.cell_size**3 / conf.mesh_size)
    return k, pk, nmodes


def delta_to_pk(delta, conf, mas="CIC"):
    spec = _spectrum(delta, conf)
    sums, _, _ = _shell_sums(spec, conf, _mas(mas))
    return _finalize(sums, conf)


def _overdensity(density, conf):
    dev = density.device
    rho = density.to(torch.float32).contiguous()
    tot = torch.zeros(1, dtype=torch.float64, device=dev)
    s = stream_handle(dev)
    call("pmb_sum", rho.data_ptr(), rho.numel(), tot.data_ptr(), s)
    delta = torch.empty_like(rho)
    call("pmb_overdensity", rho.data_ptr(), delta.data_ptr(), rho.numel(), tot.data_ptr(), s)
    return delta


def density_to_pk(density, conf, mas="CIC"):
    if conf.float_dtype == torch.float64:
        from . import x64
        return x64.density_to_pk(density, conf, _mas(mas))
    return delta_to_pk(_overdensity(density, conf), conf, mas)


def particles_to_pk(ptcl, conf, mas="CIC"):
    if conf.float_dtype == torch.float64:
        from . import x64
        return x64.particles_to_pk(ptcl, conf, _mas(mas))
    sp = SortedParticles(ptcl.pmid, ptcl.disp, conf)
    return density_to_pk(sp.scatter()[0], conf, mas)


def delta_to_cross_correlation(delta_a, delta_b, conf, mas="CIC", eps=1e-30):
    """(k, r, pk_cross, pk_a, pk_b, nmodes) (:308-345)."""
    sa = _spectrum(delta_a, conf)
    sb = _spectrum(delta_b, conf)
    pa, pb, px = _shell_sums(sa, conf, _mas(mas), sb)
    k, pk_a, n = _finalize(pa, conf)
    _, pk_b, _ = _finalize(pb, conf)
    _, pk_x, _ = _finalize(px, conf)
    r = pk_x / np.sqrt(np.maximum(pk_a * pk_b, eps))
    return k, r, pk_x, pk_a, pk_b, n


def density_to_cross_correlation(density_a, density_b, conf, mas="CIC", eps=1e-30):
    return delta_to_cross_correlation(_overdensity(density_a, conf), _overdensity(density_b, conf), conf, mas, eps)


def particles_to_cross_correlation(ptcl_a, ptcl_b, conf, mas="CIC", eps=1e-30):
    ra = SortedParticles(ptcl_a.pmid, ptcl_a.disp, conf).scatter()[0]
    rb = SortedParticles(ptcl_b.pmid, ptcl_b.disp, conf).scatter()[0]
    return density_to_cross_correlation(ra, rb, conf, mas, eps)


def cross_correlation(delta_a, delta_b, conf, mas="CIC", eps=1e-30):
    """delta_to_cross_correlation on overdensity fields (power_spectrum.py:471-490)."""
    return delta_to_cross_correlation(delta_a, delta_b, conf, mas=mas, eps=eps)


# the earlier public names of the P(k) functions (power_spectrum.py:493-496)
delta_to_quijote_pk = delta_to_pk
density_to_quijote_pk = density_to_pk
particles_to_quijote_pk = particles_to_pk


def log_binned(k, pk, nmodes, nbins=32, kmin=None, kmax=None):
    """Mode-count-weighted rebinning of integer shells into log-spaced bins."""
    kmin = k[0] if kmin is None else kmin
    kmax = k[-1] * (1 + 1e-9) if kmax is None else kmax
    edges = np.geomspace(kmin, kmax, nbins + 1)
    b = np.clip(np.searchsorted(edges, k, side='right') - 1, 0, nbins - 1)
    w = np.bincount(b, weights=nmodes, minlength=nbins)
    kb = np.bincount(b, weights=k * nmodes, minlength=nbins) / np.maximum(w, 1)
    pb = np.bincount(b, weights=pk * nmodes, minlength=nbins) / np.maximum(w, 1)
    return kb, pb, w


def pk_loss(ptcl, conf, pk_target, mas="CIC", grad=True, kmax=None):
    """L = mean_s (log P_s / P_target,s)^2 over shells with modes, and dL/d disp.

    Forward: scatter -> delta = rho/mean - 1 -> rFFT -> FP64 shell sums.
    Backward: shell-power adjoint -> C2R -> overdensity adjoint (including the
    mean) -> scatter adjoint (cic/scatter.py:386-437).  float64 particles take
    the float64 build (x64.pk_loss)."""
    if ptcl.disp.dtype == torch.float64:
        from . import x64
        return x64.pk_loss(ptcl, conf, pk_target, mas_power=_mas(mas), grad=grad, kmax=kmax)
    nx, ny, nz = conf.mesh_shape
    dev = ptcl.disp.device
    s = stream_handle(dev)
    mp = _mas(mas)
    sp = SortedParticles(ptcl.pmid, ptcl.disp, conf)
    rho = sp.scatter()[0]
    tot = torch.zeros(1, dtype=torch.float64, device=dev)
    call("pmb_sum", rho.data_ptr(), rho.numel(), tot.data_ptr(), s)
    delta = torch.empty_like(rho)
    call("pmb_overdensity", rho.data_ptr(), delta.data_ptr(), rho.numel(), tot.data_ptr(), s)
    spec = _spectrum(delta, conf)
    sums, _, _ = _shell_sums(spec, conf, mp)
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
    # dL/dP_s -> weight per shell (index 0 = shell 0 carries no loss)
    norm = conf.cell_size**3 / conf.mesh_size
    w = np.zeros(num_shells(conf))
    w[1:] = np.where(valid, 2 * lr / nv / np.where(valid, pk, 1.0), 0.0) * norm / np.maximum(nmodes, 1)
    wd = torch.from_numpy(w).to(dev)
    gspec = torch.empty_like(spec)
    call("pmb_pk_shells_adjoint", spec.data_ptr(), nx, ny, nz, _sinc_tables(conf, dev).data_ptr(), mp, len(w),
         wd.data_ptr(), 1.0, gspec.data_ptr(), s)
    fw = workspace(lib().pmb_fft_work_bytes(nx, ny, nz, 1), dev, "fft1")
    dcot = torch.empty((nx, ny, nz), dtype=torch.float32, device=dev)
    call("pmb_irfft3", nx, ny, nz, 1, gspec.data_ptr(), dcot.data_ptr(), fw.data_ptr(), s)
    # delta = rho / m - 1 with m = sum(rho)/M:  rho_cot = dcot/m - sum(dcot*rho)/(m^2 M)
    dd = torch.zeros(1, dtype=torch.float64, device=dev)
    call("pmb_dot", dcot.data_ptr(), rho.data_ptr(), rho.numel(), dd.data_ptr(), s)
    m = float(tot.item()) / rho.numel()
    shift = float(dd.item()) / (m * m * rho.numel())
    rho_cot = dcot.mul_(np.float32(1.0 / m)).sub_(np.float32(shift)).unsqueeze(0)
    disp_cot, _ = sp.interp_grad(rho_cot, u_const=float(conf.mesh_size / conf.ptcl_num))
    return loss, disp_cot
