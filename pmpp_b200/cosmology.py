"""Cosmology parameters and host-side FP64 tables.

``Cosmology`` mirrors cosmology/models.py:103-265 (A_s_1e9, n_s, Omega_m,
Omega_b, h and the optional Omega_k_, w_0_, w_a_).  ``boltzmann`` fills the
transfer and growth tables (cosmology/boltzmann.py:358-398); the growth ODE,
transfer fit, time factors and linear power are computed in FP64 by the
native library (pmpp_b200/csrc/cosmo.cpp).  The top-hat variance for sigma8
is a Simpson quadrature in ln k over the transfer-table range.
"""
from __future__ import annotations

import ctypes
import functools
import math
from dataclasses import dataclass, field, replace
from typing import Optional

import numpy as np

from ._lib import call, lib

MPC_SI = 3.0856775815e22


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


@dataclass(frozen=True, eq=False)
class Cosmology:
    conf: object = field(repr=False)
    A_s_1e9: float = 2.0
    n_s: float = 0.96
    Omega_m: float = 0.3
    Omega_b: float = 0.05
    h: float = 0.7
    Omega_k_: Optional[float] = None
    w_0_: Optional[float] = None
    w_a_: Optional[float] = None
    transfer: Optional[np.ndarray] = field(default=None, repr=False)
    growth: Optional[np.ndarray] = field(default=None, repr=False)
    growth_dOm: Optional[np.ndarray] = field(default=None, repr=False)

    @property
    def A_s(self):
        return self.A_s_1e9 * 1e-9

    @property
    def Omega_k(self):
        return 0.0 if self.Omega_k_ is None else self.Omega_k_

    @property
    def w_0(self):
        return -1.0 if self.w_0_ is None else self.w_0_

    @property
    def w_a(self):
        return 0.0 if self.w_a_ is None else self.w_a_

    @property
    def Omega_de(self):
        return 1 - (self.Omega_m + self.Omega_k)

    @property
    def k_pivot(self):
        return self.conf.k_pivot_Mpc / self.h

    def replace(self, **kw):
        return replace(self, **kw)

    @classmethod
    def from_sigma8(cls, conf, sigma8, *args, **kwargs):
        """models.py:183-203: set A_s so that sigma8(a=1) matches."""
        unit = boltzmann(cls(conf, 1.0, *args, **kwargs), conf)
        return boltzmann(cls(conf, (sigma8 / unit.sigma8)**2, *args, **kwargs), conf)

    @property
    def sigma8(self):
        """sqrt(varlin(8 Mpc/h, a=1)) (models.py:249-254)."""
        return math.sqrt(tophat_variance(8.0, self)) * float(growth(1.0, self, self.conf))

    # ---- time factors (integrator.py:114-170) ----
    def _factor(self, kind, a0, a1, a2, with_grad=False):
        conf = self.conf
        ga = np.ascontiguousarray(conf.growth_a, dtype=np.float64)
        f = ctypes.c_double()
        df = ctypes.c_double()
        call("pmb_time_factor", kind, a0, a1, a2, self.Omega_m, self.Omega_k, self.w_0, self.w_a, _p(ga), len(ga),
             _p(self.growth), _p(self.growth_dOm) if with_grad else None, ctypes.byref(f),
             ctypes.byref(df) if with_grad else None)
        return (f.value, df.value) if with_grad else f.value

    def drift_factor(self, a_vel, a_prev, a_next, with_grad=False):
        return self._factor(0, a_vel, a_prev, a_next, with_grad)

    def kick_factor(self, a_acc, a_prev, a_next, with_grad=False):
        return self._factor(1, a_acc, a_prev, a_next, with_grad)

    def lpt_factors(self, a):
        """((D1, dD1, a2HD1'), (D2, dD2, a2HD2')) and their d/d Omega_m."""
        conf = self.conf
        ga = np.ascontiguousarray(conf.growth_a, dtype=np.float64)
        out = np.zeros(6)
        dout = np.zeros(6)
        call("pmb_lpt_factors", a, self.Omega_m, self.Omega_k, self.w_0, self.w_a, _p(ga), len(ga), _p(self.growth),
             _p(self.growth_dOm), _p(out), _p(dout))
        return out.reshape(2, 3), dout.reshape(2, 3)


SimpleLCDM = functools.partial(Cosmology, A_s_1e9=2.0, n_s=0.96, Omega_m=0.3, Omega_b=0.05, h=0.7)


def transfer_fit(k, cosmo, conf=None):
    conf = cosmo.conf if conf is None else conf
    k = np.ascontiguousarray(k, dtype=np.float64)
    out = np.empty_like(k)
    call("pmb_transfer_fit", _p(k), k.size, cosmo.Omega_m, cosmo.Omega_b, cosmo.h, conf.T_cmb,
         int(conf.transfer_fit_nowiggle), _p(out))
    return out


def boltzmann(cosmo, conf=None, transfer=True, growth=True, varlin=True):
    """Transfer and growth tables (boltzmann.py:358-398); a component switched
    off stays unset.  The variance needs no table here (varlin integrates on
    demand), so ``varlin`` only mirrors the reference's signature."""
    conf = cosmo.conf if conf is None else conf
    del varlin
    T = transfer_fit(conf.transfer_k, cosmo, conf) if transfer else None
    if not growth:
        return cosmo.replace(conf=conf, transfer=T, growth=None, growth_dOm=None)
    ga = np.ascontiguousarray(conf.growth_a, dtype=np.float64)
    tab = np.zeros(6 * len(ga))
    dtab = np.zeros(6 * len(ga))
    dt0 = conf.growth_inistep[0] if isinstance(conf.growth_inistep, tuple) else conf.growth_inistep
    call("pmb_growth_table", cosmo.Omega_m, cosmo.Omega_k, cosmo.w_0, cosmo.w_a, _p(ga), len(ga), conf.a_lpt_step,
         conf.growth_rtol, conf.growth_atol, float(dt0), _p(tab), _p(dtab))
    return cosmo.replace(conf=conf, transfer=T, growth=tab.reshape(2, 3, -1), growth_dOm=dtab.reshape(2, 3, -1))


def growth(a, cosmo, conf=None, order=1, deriv=0):
    """D_m and ln-a derivatives by table interpolation (growth.py:75-111)."""
    conf = cosmo.conf if conf is None else conf
    if cosmo.growth is None:
        raise ValueError("Growth table is empty. Call boltzmann first.")
    a = np.asarray(a, dtype=np.float64)
    xp = conf.growth_a
    fp = cosmo.growth[order - 1][deriv]
    idx = np.clip(np.searchsorted(xp, a, side='right') - 1, 0, xp.shape[0] - 2)
    y = fp[idx] + (a - xp[idx]) * ((fp[idx + 1] - fp[idx]) / (xp[idx + 1] - xp[idx]))
    y = np.where(a <= xp[0], fp[0], np.where(a >= xp[-1], fp[-1], y))
    return a**order * y


def E2(a, cosmo):
    """models.py:16-50."""
    a = np.asarray(a, dtype=np.float64)
    de = a**(-3 * (1 + cosmo.w_0 + cosmo.w_a)) * np.exp(-3 * cosmo.w_a * (1 - a))
    return cosmo.Omega_m * a**-3 + cosmo.Omega_k * a**-2 + cosmo.Omega_de * de


def linear_power(k, a, cosmo, conf=None):
    """P_lin(k) [L^3] (boltzmann.py:428-484), optionally times D(a)^2."""
    conf = cosmo.conf if conf is None else conf
    if getattr(conf, "dim", 3) != 3:
        raise ValueError(f"dim={conf.dim} not supported")
    if cosmo.transfer is None:
        raise ValueError("Transfer table is empty. Call boltzmann first.")
    k = np.ascontiguousarray(k, dtype=np.float64)
    out = np.empty_like(k)
    tk = np.ascontiguousarray(conf.transfer_k, dtype=np.float64)
    tt = np.ascontiguousarray(cosmo.transfer, dtype=np.float64)
    call("pmb_linear_power", _p(k), k.size, _p(tk), _p(tt), len(tk), cosmo.A_s, cosmo.n_s, cosmo.Omega_m, cosmo.h,
         conf.k_pivot_Mpc, _p(out))
    if a is not None:
        out = out * growth(a, cosmo, conf)**2
    return out


def tophat_variance(R, cosmo, conf=None):
    """sigma^2(R) without growth by Simpson quadrature in ln k."""
    conf = cosmo.conf if conf is None else conf
    tk = conf.transfer_k
    lnk = np.linspace(np.log(tk[1]), np.log(tk[-1]), 2**16 + 1)
    k = np.exp(lnk)
    P = linear_power(k, None, cosmo, conf)
    x = k * R
    W = 3 * (np.sin(x) - x * np.cos(x)) / x**3
    f = k**3 * P / (2 * np.pi**2) * W**2
    h = lnk[1] - lnk[0]
    return h / 3 * (f[0] + f[-1] + 4 * f[1:-1:2].sum() + 2 * f[2:-1:2].sum())


def transfer(k, cosmo, conf=None):
    """Matter transfer function at k [1/L], interpolated in the table that
    boltzmann fills (boltzmann.py:140-174)."""
    conf = cosmo.conf if conf is None else conf
    if cosmo.transfer is None:
        raise ValueError("Transfer table is empty. Call boltzmann first.")
    k = np.asarray(k)
    dtype = np.promote_types(k.dtype, np.float64)
    return np.interp(k, conf.transfer_k, cosmo.transfer).astype(dtype)


def varlin(R, a, cosmo, conf=None):
    """Linear matter variance sigma^2(R) at scales R [L], times D(a)^2 unless a
    is None (boltzmann.py:314-355).  Each R is evaluated by the Simpson
    quadrature of tophat_variance rather than interpolated in a table."""
    conf = cosmo.conf if conf is None else conf
    if cosmo.transfer is None or (a is not None and cosmo.growth is None):
        raise ValueError("Linear matter overdensity variance table is empty. Call boltzmann first.")
    R = np.asarray(R, dtype=np.float64)
    s2 = np.vectorize(lambda r: tophat_variance(float(r), cosmo, conf), otypes=[np.float64])(R)
    if a is not None:
        s2 = s2 * np.asarray(growth(a, cosmo, conf), dtype=np.float64)**2
    return s2


def cosmology_param_names(cosmo):
    """Differentiable parameter names of this instance (models.py:267-288):
    the five base parameters and each optional one that is set."""
    names = ["A_s_1e9", "n_s", "Omega_m", "Omega_b", "h"]
    names += [n for n in ("Omega_k_", "w_0_", "w_a_") if getattr(cosmo, n) is not None]
    return tuple(names)


def cosmology_param_values(cosmo, names=None):
    """Parameter values in the order of names (default cosmology_param_names)
    (models.py:291-309)."""
    names = cosmology_param_names(cosmo) if names is None else names
    return tuple(getattr(cosmo, n) for n in names)


def replace_cosmology_params(cosmo, names, values):
    """A cosmology with the named parameters replaced (models.py:312-329)."""
    return cosmo.replace(**dict(zip(names, values)))


def _touch():
    lib()
