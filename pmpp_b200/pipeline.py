"""The differentiable forward model: white noise -> linear modes -> 2LPT ->
KDK N-body -> P(k) loss, and its hand-written reverse pass.

This is the composition of initial_conditions/modes.py (linear_modes),
initial_conditions/lpt.py (lpt), nbody/solver.py (nbody with its custom VJP)
and analysis/power_spectrum.py that a PM++ user differentiates with jax.grad;
here the reverse pass chains the hand-written adjoints: P(k) loss adjoint ->
nbody_adj (reverse sweep with recomputation) -> lpt adjoint -> linear-mode
amplitude.  Gradients: the white-noise modes (packed dL/dRe + i dL/dIm),
Omega_m and the amplitude (A_s_1e9, or sigma8 when the cosmology was built
with ``Cosmology.from_sigma8``).
"""
from __future__ import annotations

import numpy as np
import torch

from . import lpt as _lpt
from . import modes as _modes
from . import power_spectrum as _ps
from .cosmology import Cosmology, boltzmann
from .nbody import NBodyRun
from .particles import Particles


class ForwardModel:
    def __init__(self, conf, cosmo, correction=None):
        self.conf = conf
        self.cosmo = cosmo
        self.correction = correction

    def forward(self, omega):
        """omega: white-noise rFFT modes on the particle grid.  Returns final particles."""
        conf, cosmo = self.conf, self.cosmo
        self.omega = omega
        self.amp = _modes.linear_amplitude(cosmo, conf, device=omega.device)
        lin = _modes.linear_modes(omega, cosmo, conf)
        self.lpt = _lpt.lpt_full(lin, cosmo, conf)
        self.run = NBodyRun(conf, cosmo, self.correction)
        self.final = self.run.forward(self.lpt.ptcl)
        return self.final

    def loss(self, pk_target, grad=True):
        return _ps.pk_loss(self.final, self.conf, pk_target, grad=grad)

    def backward(self, disp_cot, vel_cot=None):
        """Reverse pass from final-state cotangents.

        Returns dict(modes=complex tensor, Omega_m=float, A_s_1e9=float)."""
        conf, cosmo = self.conf, self.cosmo
        z = torch.zeros_like(disp_cot)
        cot = Particles(conf, self.final.pmid, disp_cot, z if vel_cot is None else vel_cot, z.clone())
        _, c0, om_nbody = self.run.adjoint(self.final, cot)
        # LPT adjoint to the linear modes; the white-noise cotangent follows by
        # the (real) linear-mode amplitude, the parameter cotangents from mc_lin
        mc_lin, om_lpt = _lpt.lpt_vjp(self.lpt, c0.disp, c0.vel, cosmo, conf)
        mc_noise = mc_lin * self.amp
        if conf.float_dtype == torch.float64:
            from . import x64
            dAs, om_lin = x64.linear_modes_param_cotangents(self.omega, mc_lin, cosmo, conf)
        else:
            dAs, om_lin = _modes.linear_modes_param_cotangents(self.omega, mc_lin, cosmo, conf)
        return {"modes": mc_noise, "Omega_m": om_nbody + om_lpt + om_lin, "A_s_1e9": dAs,
                "Omega_m_parts": (om_nbody, om_lpt, om_lin)}


def sigma8_chain(grads, cosmo, conf, h=1e-4):
    """Convert (dL/dA_s, dL/dOmega_m at fixed A_s) to (dL/dsigma8, dL/dOmega_m at
    fixed sigma8) for A_s = (sigma8 / sigma8_unit(Omega_m))^2 (models.py:183-203)."""
    s8 = cosmo.sigma8
    kw = dict(n_s=cosmo.n_s, Omega_b=cosmo.Omega_b, h=cosmo.h)
    su = lambda om: boltzmann(Cosmology(conf, 1.0, Omega_m=om, **kw), conf).sigma8
    dlnsu = (np.log(su(cosmo.Omega_m + h)) - np.log(su(cosmo.Omega_m - h))) / (2 * h)
    A = cosmo.A_s_1e9
    d_sigma8 = grads["A_s_1e9"] * 2 * A / s8
    d_om = grads["Omega_m"] + grads["A_s_1e9"] * (-2 * A * dlnsu)
    return d_sigma8, d_om
