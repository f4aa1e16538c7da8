"""Potential corrections applied inside the PM force.

* ``PMWindowCompensation`` -- the analytic CIC-window compensation
  (corrections/window.py:23-265): gain = W(k)^(-order*windows*alpha) capped at
  max_gain, tapered to 1 between taper_start and taper_stop of the particle
  Nyquist wavenumber, with the discrete-Laplacian Green's function.  Evaluated
  once per configuration into a device transfer table.
* ``LearnedGreen`` -- a width-64 sin-MLP T(|k|, a, Omega_m, sigma8) = 1 + f(x)
  (bf16 weights, FP32 accumulation) evaluated by pmb_mlp_table on the table of
  integer |n|^2 each force evaluation and trained through the hand-written
  adjoints (pmb_transfer_cot + pmb_mlp_backward), Adam in FP32.  The reference's
  learned radial filter (corrections/radial.py:29-216) is a spline whose knots
  come from a sin-MLP of a only; this network takes the cosmology as input.

Both follow the protocol pmpp_b200.gravity expects: ``green_kernel`` and
``transfer_tables(a, cosmo, conf) -> (transfer or None, radial or None)``.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from ._lib import call, lib
from .runtime import stream_handle


class PMWindowCompensation:
    """corrections/window.py:23-265 (PMWindowCompensationCorrection): transfer
    gain W(k)^(-order*windows*alpha) capped and tapered, the Green's function
    ("continuum" or "discrete_laplacian") and the force derivative
    ("spectral" or FastPM's "fastpm_4point"); interlacing selects the
    interlaced force (two deposits, gravity.py:446-463)."""

    green_kernel = 1  # discrete Laplacian (window.py:100-108 default)

    def __init__(self, alpha=0.48, max_gain=4.0, assignment_order=2, windows=2, taper_start=0.75, taper_stop=1.0,
                 green_kernel="discrete_laplacian", gradient_kernel="spectral", interlacing=False):
        if green_kernel not in ("continuum", "discrete_laplacian"):
            raise ValueError(f"Unsupported PM Green's function {green_kernel!r}.")
        if gradient_kernel not in ("spectral", "fastpm_4point"):
            raise ValueError(f"Unsupported force-gradient kernel {gradient_kernel!r}.")
        self.alpha = alpha
        self.max_gain = max_gain
        self.assignment_order = assignment_order
        self.windows = windows
        self.taper_start = taper_start
        self.taper_stop = taper_stop
        self.green_kernel = 1 if green_kernel == "discrete_laplacian" else 0
        self.gradient_kernel = gradient_kernel
        self.interlacing = bool(interlacing)
        self._cache = {}

    def transfer_tables(self, a, cosmo, conf):
        """Gain per half-spectrum cell in the configuration's float dtype."""
        if self.alpha == 0:
            return None, None  # gain W^0 = 1 everywhere: no transfer
        dev = conf.device
        key = (conf.mesh_shape, conf.cell_size, conf.ptcl_spacing, str(dev), str(conf.float_dtype))
        if key not in self._cache:
            f = conf.np_dtype.type
            kx, ky, kz = [torch.from_numpy(k.astype(conf.np_dtype)).to(dev) for k in conf.kvec]
            c = f(conf.cell_size)
            two_pi = f(2 * np.pi)
            sinc = lambda x: torch.where(x == 0, torch.ones_like(x), torch.sin(np.pi * x) / (np.pi * x))
            sx = sinc(kx * c / two_pi)[:, None, None]
            sy = sinc(ky * c / two_pi)[None, :, None]
            sz = sinc(kz * c / two_pi)[None, None, :]
            base = torch.clamp((sx * sy * sz).abs(), min=1e-6)
            gain = base**(-float(self.assignment_order * self.windows * self.alpha))
            if self.max_gain is not None and self.max_gain > 0:
                gain = torch.clamp(gain, max=float(self.max_gain))
            if self.taper_stop > self.taper_start:
                kn = f(np.pi / conf.ptcl_spacing)
                q = torch.maximum(torch.maximum(kx.abs()[:, None, None], ky.abs()[None, :, None]),
                                  kz.abs()[None, None, :]) / kn
                t = torch.clamp((q - self.taper_start) / (self.taper_stop - self.taper_start), 0.0, 1.0)
                gain = 1.0 + (gain - 1.0) * (1.0 - t * t * (3.0 - 2.0 * t))
            self._cache[key] = gain.to(conf.float_dtype).contiguous()
        return self._cache[key], None


class PGDPotentialCorrection:
    """FastPM-style PGD residual potential as a multiplicative transfer
    (corrections/pgd.py:14-35, 154-237): T(k, a) = 1 - alpha(a) band(k) with
    alpha(a) = alpha0 10^(A a^2 - B a) and band = exp(-kl^2/k^2 - k^4/ks^4)
    (0 at k = 0), evaluated in float32 per scale factor."""

    green_kernel = 0
    gradient_kernel = "spectral"

    def __init__(self, alpha0=0.1, A=0.0, B=0.0, kl=0.1, ks=1.0):
        self.alpha0, self.A, self.B, self.kl, self.ks = alpha0, A, B, kl, ks
        self._cache = {}

    def alpha(self, a, f=np.float32):
        return f(self.alpha0) * (f(10.0)**(f(self.A) * f(a)**2 - f(self.B) * f(a)))

    def transfer_tables(self, a, cosmo, conf):
        """Transfer per half-spectrum cell at scale factor a, in the
        configuration's float dtype."""
        a = 1.0 if a is None else float(a)
        key = (a, conf.mesh_shape, conf.cell_size, str(conf.device), str(conf.float_dtype))
        if key not in self._cache:
            if len(self._cache) > 64:
                self._cache.clear()
            dev = conf.device
            f = conf.np_dtype.type
            kx, ky, kz = [torch.from_numpy(k.astype(conf.np_dtype)).to(dev) for k in conf.kvec]
            k2 = (kx[:, None, None]**2 + ky[None, :, None]**2) + kz[None, None, :]**2
            safe = torch.where(k2 > 0, k2, torch.ones_like(k2))
            band = torch.exp(-f(self.kl)**2 / safe - safe**2 / f(self.ks)**4)
            band = torch.where(k2 > 0, band, torch.zeros_like(band))
            self._cache[key] = (1.0 - float(self.alpha(a, f)) * band).to(conf.float_dtype).contiguous()
        return self._cache[key], None


class HighKSofteningCorrection:
    """High-k spectral softening (corrections/softening.py:12-80): T = max(1 -
    strength taper(q), 0) with q = max_i |k_i| / k_Ny(particles) and taper the
    smoothstep (or linear) ramp from start to stop."""

    green_kernel = 0
    gradient_kernel = "spectral"

    def __init__(self, strength=0.0, start=0.7, stop=1.0, mode="smoothstep"):
        if mode not in ("smoothstep", "linear"):
            raise ValueError(f"Unsupported high-k softening mode {mode!r}.")
        self.strength, self.start, self.stop, self.mode = strength, start, stop, mode
        self._cache = {}

    def transfer_tables(self, a, cosmo, conf):
        """Transfer per half-spectrum cell in the configuration's float dtype."""
        key = (conf.mesh_shape, conf.cell_size, conf.ptcl_spacing, str(conf.device), str(conf.float_dtype))
        if key not in self._cache:
            dev = conf.device
            f = conf.np_dtype.type
            kx, ky, kz = [torch.from_numpy(k.astype(conf.np_dtype)).to(dev).abs() for k in conf.kvec]
            kn = f(np.pi / conf.ptcl_spacing)
            q = torch.maximum(torch.maximum(kx[:, None, None] / kn, ky[None, :, None] / kn), kz[None, None, :] / kn)
            t = torch.clamp((q - f(self.start)) / max(f(self.stop - self.start), f(1e-6)), 0.0, 1.0)
            taper = t * t * (3.0 - 2.0 * t) if self.mode == "smoothstep" else t
            self._cache[key] = torch.clamp(1.0 - f(self.strength) * taper, min=0.0).to(conf.float_dtype)
        return self._cache[key], None


class CombinedPotentialCorrection:
    """Several corrections at once (corrections/core.py:286-334, combined.py):
    the product of their transfers, the first non-continuum Green's function and
    the one non-spectral force derivative they ask for."""

    def __init__(self, window=None, pgd=None, softening=None, radial=None, mesh_cnn=None):
        self.parts = [c for c in (window, pgd, softening, radial, mesh_cnn) if c is not None]
        self.mesh_cnn_part = mesh_cnn
        self.green_kernel = next((c.green_kernel for c in self.parts if getattr(c, "green_kernel", 0) != 0), 0)
        grads = {getattr(c, "gradient_kernel", "spectral") for c in self.parts} - {"spectral"}
        if len(grads) > 1:
            raise ValueError(f"Combined correction requests incompatible force-gradient kernels: {sorted(grads)!r}.")
        self.gradient_kernel = next(iter(grads), "spectral")

    def transfer_tables(self, a, cosmo, conf):
        T, R = None, None
        for c in self.parts:
            t, r = c.transfer_tables(a, cosmo, conf)
            if t is not None:
                T = t if T is None else T * t
            if r is not None:
                if R is not None:
                    raise ValueError("at most one radial table per combined correction")
                R = r
        return (None if T is None else T.contiguous()), R


def _window_from(kw):
    """init_pm_window_compensation_correction's keywords and aliases (corrections/window.py:159-177)."""
    return PMWindowCompensation(
        alpha=kw.get("alpha", kw.get("window_alpha", 0.48)), max_gain=kw.get("max_gain", kw.get("window_max_gain", 4.0)),
        assignment_order=kw.get("assignment_order", 2), windows=kw.get("windows", 2),
        taper_start=kw.get("taper_start", kw.get("window_taper_start", 0.75)),
        taper_stop=kw.get("taper_stop", kw.get("window_taper_stop", 1.0)), interlacing=kw.get("interlacing", False),
        green_kernel=kw.get("green_kernel", "discrete_laplacian"),
        gradient_kernel=kw.get("gradient_kernel", kw.get("window_gradient_kernel", "spectral")))


def _pgd_from(kw):
    """init_pgd_potential_correction's keywords and aliases (corrections/pgd.py:88-104)."""
    return PGDPotentialCorrection(alpha0=kw.get("alpha0", kw.get("pgd_alpha0", 0.1)), A=kw.get("A", kw.get("pgd_A", 0.0)),
                                  B=kw.get("B", kw.get("pgd_B", 0.0)), kl=kw.get("kl", kw.get("pgd_kl", 0.1)),
                                  ks=kw.get("ks", kw.get("pgd_ks", 1.0)))


def _softening_from(kw):
    """init_high_k_softening_correction's keywords and aliases (corrections/softening.py:32-46)."""
    return HighKSofteningCorrection(strength=kw.get("strength", kw.get("softening_strength", 0.0)),
                                    start=kw.get("start", kw.get("softening_start", 0.7)),
                                    stop=kw.get("stop", kw.get("softening_stop", 1.0)),
                                    mode=kw.get("mode", kw.get("softening_mode", "smoothstep")))


def _mesh_cnn_from(kw):
    """init_mesh_cnn_potential_correction's keywords (corrections/mesh_cnn.py:158-205,
    the mesh_* aliases of corrections/core.py:28-37)."""
    from .meshcnn import MeshCNNCorrection
    return MeshCNNCorrection(channels=kw.get("channels", kw.get("mesh_channels", 8)),
                             depth=kw.get("depth", kw.get("mesh_depth", 4)),
                             max_residual=kw.get("max_residual", kw.get("mesh_max_residual", 0.1)),
                             output_init_scale=kw.get("output_init_scale", kw.get("mesh_output_init_scale", 1e-2)),
                             seed=kw.get("seed", 0), device=kw.get("device", "cuda"),
                             sigma8_value=kw.get("sigma8_value", 0.8),
                             allow_missing_sigma8=kw.get("allow_missing_sigma8", False))


def init_potential_correction(model, **kwargs):
    """The analytic models of init_potential_correction (corrections/core.py:40-151):
    "pm_window" / "cic_compensation" / "cic_window_compensation" (the window
    compensation), "fastpm_1_4" (continuum Green's function) and "fastpm_3_4"
    (discrete Laplacian), both with FastPM's 4-point gradient and no window
    gain, "pgd" / "fastpm_pgd", "high_k_softening" / "softening" /
    "fastpm_softening", and the window combined with either ("windowed_pgd",
    "pm_window+pgd", "pgd_window", "windowed_softening", "pm_window+softening"), the
    mesh CNN ("mesh_cnn", "cnn") and the window with it ("windowed_mesh_cnn",
    "pm_window+mesh_cnn").  The trainable window / PGD variants and the radial
    spline (LearnedGreen stands in for it) are not built."""
    kw = dict(kwargs)
    kw.pop("dtype", None)
    if model in ("pm_window", "cic_compensation", "cic_window_compensation"):
        return _window_from(kw)
    if model in ("fastpm_1_4", "fastpm_3_4"):
        kw.update(window_alpha=0.0, alpha=0.0, gradient_kernel="fastpm_4point",
                  green_kernel="continuum" if model == "fastpm_1_4" else "discrete_laplacian")
        return _window_from(kw)
    if model in ("pgd", "fastpm_pgd"):
        return _pgd_from(kw)
    if model in ("high_k_softening", "softening", "fastpm_softening"):
        return _softening_from(kw)
    if model in ("windowed_pgd", "pm_window+pgd", "pgd_window"):
        return CombinedPotentialCorrection(window=_window_from(kw), pgd=_pgd_from(kw))
    if model in ("windowed_softening", "pm_window+softening"):
        return CombinedPotentialCorrection(window=_window_from(kw), softening=_softening_from(kw))
    if model in ("mesh_cnn", "cnn"):
        return _mesh_cnn_from(kw)
    if model in ("windowed_mesh_cnn", "pm_window+mesh_cnn"):
        return CombinedPotentialCorrection(window=_window_from(kw), mesh_cnn=_mesh_cnn_from(kw))
    raise ValueError(f"Unsupported correction model {model!r}.")


def radial_table_len(conf):
    nx, ny, nz = conf.mesh_shape
    return (nx // 2)**2 + (ny // 2)**2 + (nz // 2)**2 + 1


class LearnedGreen:
    """Trainable multiplicative Green's-function correction."""

    green_kernel = 0
    trainable = True

    def __init__(self, device="cuda", seed=0, sigma8=0.8, init_scale=1.0):
        nw, nb = ctypes.c_int(), ctypes.c_int()
        call("pmb_mlp_param_counts", ctypes.byref(nw), ctypes.byref(nb))
        self.n_weights, self.n_biases = nw.value, nb.value
        H = 64
        g = torch.Generator().manual_seed(seed)
        u = lambda shape, fan: (torch.rand(shape, generator=g) * 2 - 1) * math.sqrt(6.0 / fan) * init_scale
        W1 = u((H, 4), 4)
        W2 = u((H, H), H)
        W3 = u((H, H), H)
        W4 = torch.zeros(H)  # T = 1 at initialisation: starts from the plain Green's function
        self.w = torch.cat([W1.reshape(-1), W2.reshape(-1), W3.reshape(-1), W4]).to(device)
        self.b = torch.cat([u((H, ), 4), u((H, ), H), u((H, ), H), torch.zeros(1)]).to(device)
        assert self.w.numel() == self.n_weights and self.b.numel() == self.n_biases
        self.device = torch.device(device)
        self.sigma8 = sigma8
        self.grad = torch.zeros(self.n_weights + self.n_biases, dtype=torch.float32, device=device)
        self._adam = None
        self._sync_bf16()

    def _sync_bf16(self):
        self.w16 = self.w.to(torch.bfloat16).contiguous()

    def parameters(self):
        return torch.cat([self.w, self.b])

    def load_parameters(self, p):
        p = p.to(self.device, torch.float32)
        self.w = p[:self.n_weights].clone()
        self.b = p[self.n_weights:].clone()
        self._sync_bf16()

    def _kscale(self, conf):
        return 2.0 / conf.mesh_shape[0]

    def _cond(self, a, cosmo, conf):
        s8 = cosmo.__dict__.get("_sigma8_cached")
        if s8 is None:
            s8 = float(cosmo.sigma8) if cosmo.transfer is not None and cosmo.growth is not None else self.sigma8
            object.__setattr__(cosmo, "_sigma8_cached", s8)
        return float(self._kscale(conf)), float(a), float(cosmo.Omega_m), float(s8)

    def table(self, a, cosmo, conf):
        L = radial_table_len(conf)
        out = torch.empty(L, dtype=torch.float32, device=self.device)
        ks, aa, om, s8 = self._cond(a, cosmo, conf)
        call("pmb_mlp_table", self.w16.data_ptr(), self.b.data_ptr(), ks, aa, om, s8, L, out.data_ptr(),
             stream_handle(self.device))
        return out

    def transfer_tables(self, a, cosmo, conf):
        if conf.mesh_shape[0] != conf.mesh_shape[1] or conf.mesh_shape[0] != conf.mesh_shape[2]:
            raise ValueError("LearnedGreen needs a cubic force mesh")
        return None, self.table(a, cosmo, conf)

    def accumulate(self, a, cosmo, conf, table_cot):
        """grad += d(sum_n table_cot[n] T_n) / d params for one force evaluation."""
        ks, aa, om, s8 = self._cond(a, cosmo, conf)
        call("pmb_mlp_backward", self.w16.data_ptr(), self.b.data_ptr(), ks, aa, om, s8, int(table_cot.numel()),
             table_cot.data_ptr(), self.grad.data_ptr(), stream_handle(self.device))

    def zero_grad(self):
        self.grad.zero_()

    def adam_step(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8, clip=None):
        """Adam in FP32 on the master parameters; bf16 copies refreshed after."""
        p = self.parameters()
        g = self.grad.clone()
        if clip is not None:
            n = float(g.norm())
            if n > clip:
                g *= clip / n
        if self._adam is None:
            self._adam = [torch.zeros_like(p), torch.zeros_like(p), 0]
        m, v, t = self._adam
        t += 1
        m.mul_(b1).add_(g, alpha=1 - b1)
        v.mul_(b2).addcmul_(g, g, value=1 - b2)
        mh = m / (1 - b1**t)
        vh = v / (1 - b2**t)
        p = p - lr * mh / (vh.sqrt() + eps)
        self._adam = [m, v, t]
        self.load_parameters(p)
