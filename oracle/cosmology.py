"""CPU oracle -- test infrastructure only, never part of the product path.

FP64 NumPy restatement of PM++'s host-side cosmology: E^2(a), dlnH/dlna,
Omega_m(a), the Eisenstein-Hu transfer fit, the growth ODE integrated with the
same adaptive Dormand-Prince scheme, growth-table interpolation, the linear
power spectrum and the top-hat variance used for sigma8.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
import this module.  Each function cites the reference file:line it restates
(paths relative to the PM++ source tree).

Parity status: the growth ODE, transfer fit and linear power follow the
reference formulas exactly; the sigma8 top-hat variance is a direct quadrature
instead of the reference's third-party ``mcfit.TophatVar`` (FFTLog), so the
absolute sigma8 normalisation is *parity unpinned* (agreement ~1e-4).
"""
from __future__ import annotations

import math

import numpy as np

# Unit system, src/pmpp/core/configuration.py:199-209 and :484-506.
M_SUN_SI = 1.98847e30
MPC_SI = 3.0856775815e22
H0_SI = 1e5 / MPC_SI
C_SI = 299792458
G_SI = 6.67430e-11
UNIT_M = 1e10 * M_SUN_SI
UNIT_L = MPC_SI
UNIT_T = 1 / H0_SI
UNIT_V = UNIT_L / UNIT_T
H_0 = H0_SI * UNIT_T
C_LIGHT = C_SI / UNIT_V


class Cosmo:
    """Cosmological parameters (src/pmpp/cosmology/models.py:103-265)."""

    def __init__(self, A_s_1e9=2.0, n_s=0.96, Omega_m=0.3, Omega_b=0.05, h=0.7, Omega_k=0.0, w_0=-1.0, w_a=0.0):
        self.A_s_1e9 = A_s_1e9
        self.n_s = n_s
        self.Omega_m = Omega_m
        self.Omega_b = Omega_b
        self.h = h
        self.Omega_k = Omega_k
        self.w_0 = w_0
        self.w_a = w_a
        self.transfer = None
        self.growth = None

    @property
    def A_s(self):
        return self.A_s_1e9 * 1e-9

    @property
    def Omega_c(self):
        return self.Omega_m - self.Omega_b

    @property
    def Omega_de(self):
        return 1 - (self.Omega_m + self.Omega_k)

    def k_pivot(self, k_pivot_Mpc=0.05):
        # models.py:211-217
        return k_pivot_Mpc / (self.h * MPC_SI) * UNIT_L

    def replace(self, **kw):
        c = Cosmo(self.A_s_1e9, self.n_s, self.Omega_m, self.Omega_b, self.h, self.Omega_k, self.w_0, self.w_a)
        for k, v in kw.items():
            setattr(c, k, v)
        return c


def E2(a, cosmo):
    """models.py:16-50."""
    a = np.asarray(a)
    de_a = a**(-3 * (1 + cosmo.w_0 + cosmo.w_a)) * np.exp(-3 * cosmo.w_a * (1 - a))
    return cosmo.Omega_m * a**-3 + cosmo.Omega_k * a**-2 + cosmo.Omega_de * de_a


def _dE2_da(a, cosmo):
    p = -3 * (1 + cosmo.w_0 + cosmo.w_a)
    q = -3 * cosmo.w_a
    de_a = a**p * np.exp(q * (1 - a))
    return -3 * cosmo.Omega_m * a**-4 - 2 * cosmo.Omega_k * a**-3 + cosmo.Omega_de * de_a * (p / a - q)


def H_deriv(a, cosmo):
    """dlnH/dlna = a E2'(a) / (2 E2), models.py:53-73."""
    return 0.5 * a * _dE2_da(a, cosmo) / E2(a, cosmo)


def Omega_m_a(a, cosmo):
    """models.py:76-100."""
    return cosmo.Omega_m / (a**3 * E2(a, cosmo))


# --------------------------------------------------------------------------
# Adaptive Dormand-Prince integration, restating the scheme of
# src/pmpp/numerics/ode.py:90-422 (tableau, error norm, step control and the
# quartic dense output at requested times).  The complex dtype is allowed so
# the same step sequence can carry complex-step tangents (step control only
# looks at real parts).
# --------------------------------------------------------------------------
_ALPHA = np.array([1 / 5, 3 / 10, 4 / 5, 8 / 9, 1., 1., 0])
_BETA = np.array([[1 / 5, 0, 0, 0, 0, 0, 0], [3 / 40, 9 / 40, 0, 0, 0, 0, 0], [44 / 45, -56 / 15, 32 / 9, 0, 0, 0, 0],
                  [19372 / 6561, -25360 / 2187, 64448 / 6561, -212 / 729, 0, 0, 0],
                  [9017 / 3168, -355 / 33, 46732 / 5247, 49 / 176, -5103 / 18656, 0, 0],
                  [35 / 384, 0, 500 / 1113, 125 / 192, -2187 / 6784, 11 / 84, 0]])
_C_SOL = np.array([35 / 384, 0, 500 / 1113, 125 / 192, -2187 / 6784, 11 / 84, 0])
_C_ERR = np.array([
    35 / 384 - 1951 / 21600, 0, 500 / 1113 - 22642 / 50085, 125 / 192 - 451 / 720, -2187 / 6784 - -12231 / 42400,
    11 / 84 - 649 / 6300, -1. / 60.
])
_C_MID = np.array([
    6025192743 / 30085553152 / 2, 0, 51252292925 / 65400821598 / 2, -2691868925 / 45128329728 / 2,
    187940372067 / 1594534317056 / 2, -1776094331 / 19743644256 / 2, 11237099 / 235043384 / 2
])


def _rk_step(fun, y0, f0, t0, dt):
    k = np.zeros((7, y0.shape[0]), dtype=y0.dtype)
    k[0] = f0
    for i in range(1, 7):
        ti = t0 + dt * _ALPHA[i - 1]
        yi = y0 + dt * (_BETA[i - 1] @ k)
        k[i] = fun(yi, ti)
    y1 = dt * (_C_SOL @ k) + y0
    err = dt * (_C_ERR @ k)
    return y1, k[-1], err, k


def _interp_fit(y0, y1, k, dt):
    y_mid = y0 + dt * (_C_MID @ k)
    dy0, dy1 = k[0], k[-1]
    a = -2. * dt * dy0 + 2. * dt * dy1 - 8. * y0 - 8. * y1 + 16. * y_mid
    b = 5. * dt * dy0 - 3. * dt * dy1 + 18. * y0 + 14. * y1 - 32. * y_mid
    c = -4. * dt * dy0 + dt * dy1 - 11. * y0 - 5. * y1 + 16. * y_mid
    d = dt * dy0
    e = y0
    return [a, b, c, d, e]


def odeint(fun, y0, ts, rtol, atol, dt0=1.0, mxstep=np.inf):
    """Dense-output DOPRI5 integration at times ``ts`` (ode.py:351-422)."""
    y = np.asarray(y0).copy()
    f = fun(y, ts[0])
    t = float(ts[0])
    dt = float(dt0)
    last_t = t
    coeff = [y.copy() for _ in range(5)]
    out = [y.copy()]
    for target in ts[1:]:
        i = 0
        while t < target and i < mxstep and dt > 0:
            ny, nf, nerr, k = _rk_step(fun, y, f, t, dt)
            nt = t + dt
            tol = atol + rtol * np.maximum(np.abs(y.real), np.abs(ny.real))
            ratio = math.sqrt(float(np.mean((nerr.real / tol)**2)))
            ncoeff = _interp_fit(y, ny, k, dt)
            # optimal_step_size, ode.py:275-301
            dfactor = 1.0 if ratio < 1 else 0.2
            if ratio == 0:
                ndt = dt * 10.0
            else:
                ndt = dt * min(10.0, max(ratio**(-1.0 / 5.0) * 0.9, dfactor))
            ndt = max(ndt, 0.0)
            i += 1
            if ratio <= 1.0:
                y, f, last_t, t, coeff = ny, nf, t, nt, ncoeff
            dt = ndt
        x = (target - last_t) / (t - last_t)
        yt = coeff[0]
        for c in coeff[1:]:
            yt = yt * x + c
        out.append(yt)
    return np.stack(out)


# --------------------------------------------------------------------------
# Transfer function, boltzmann.py:33-137.
# --------------------------------------------------------------------------
def transfer_fit(k, cosmo, T_cmb=2.7255, nowiggle=False):
    k = np.asarray(k, dtype=np.result_type(k, float, cosmo.Omega_m))
    k = k * cosmo.h / UNIT_L * MPC_SI
    T2_cmb_norm = (T_cmb / 2.7)**2
    h2 = cosmo.h**2
    w_m = cosmo.Omega_m * h2
    w_b = cosmo.Omega_b * h2
    zero_baryon = w_b <= 0
    w_b_safe = 1e-8 if zero_baryon else w_b
    f_b = cosmo.Omega_b / cosmo.Omega_m
    f_c = cosmo.Omega_c / cosmo.Omega_m
    z_eq = 2.50e4 * w_m / T2_cmb_norm**2
    k_eq = 7.46e-2 * w_m / T2_cmb_norm
    b1 = 0.313 * w_m**-0.419 * (1 + 0.607 * w_m**0.674)
    b2 = 0.238 * w_m**0.223
    z_d = 1291 * w_m**0.251 / (1 + 0.659 * w_m**0.828) * (1 + b1 * w_b**b2)
    R_d = 31.5 * w_b_safe / T2_cmb_norm**2 * (1e3 / z_d)
    R_eq = 31.5 * w_b_safe / T2_cmb_norm**2 * (1e3 / z_eq)
    s = (2 / (3 * k_eq) * np.sqrt(6 / R_eq) * np.log((np.sqrt(1 + R_d) + np.sqrt(R_eq + R_d)) / (1 + np.sqrt(R_eq))))
    k_silk = 1.6 * w_b**0.52 * w_m**0.73 * (1 + (10.4 * w_m)**-0.95)
    if nowiggle:
        alpha_gamma = (1 - 0.328 * np.log(431 * w_m) * f_b + 0.38 * np.log(22.3 * w_m) * f_b**2)
        gamma_eff_ratio = alpha_gamma + (1 - alpha_gamma) / (1 + (0.43 * k * s)**4)
        q_eff = k / (13.41 * k_eq * gamma_eff_ratio)
        L0 = np.log(2 * np.e + 1.8 * q_eff)
        C0 = 14.2 + 731 / (1 + 62.5 * q_eff)
        return L0 / (L0 + C0 * q_eff**2)
    a1 = (46.9 * w_m)**0.670 * (1 + (32.1 * w_m)**-0.532)
    a2 = (12.0 * w_m)**0.424 * (1 + (45.0 * w_m)**-0.582)
    alpha_c = a1**-f_b * a2**-f_b**3
    b1 = 0.944 / (1 + (458 * w_m)**-0.708)
    b2 = (0.395 * w_m)**-0.0266
    beta_c = 1 / (1 + b1 * (f_c**b2 - 1))

    def T0_tilde(k, alpha_c, beta_c):
        q = k / (13.41 * k_eq)
        L = np.log(np.e + 1.8 * beta_c * q)
        C = 14.2 / alpha_c + 386 / (1 + 69.9 * q**1.08)
        return L / (L + C * q**2)

    T_no_baryon = T0_tilde(k, 1, 1)
    f = 1 / (1 + (k * s / 5.4)**4)
    T_c = f * T0_tilde(k, 1, beta_c) + (1 - f) * T0_tilde(k, alpha_c, beta_c)
    y = (1 + z_eq) / (1 + z_d)
    x = np.sqrt(1 + y)
    G = y * (-6 * x + (2 + 3 * y) * np.log((x + 1) / (x - 1)))
    alpha_b = 2.07 * k_eq * s * (1 + R_d)**-0.75 * G
    beta_node = 8.41 * w_m**0.435
    beta_b = 0.5 + f_b + (3 - 2 * f_b) * np.sqrt(1 + (17.2 * w_m)**2)
    ks = k * s
    # jnp.sinc(x) = sin(pi x)/(pi x), same definition as np.sinc
    sinc = np.sinc(ks**2 / (np.pi * np.cbrt(beta_node**3 + ks**3)))
    T_b = (T0_tilde(k, 1, 1) / (1 + (ks / 5.2)**2) + alpha_b * ks**3 / (beta_b**3 + ks**3) * np.exp(-(k / k_silk)**1.4)) * sinc
    return T_no_baryon if zero_baryon else f_c * T_c + f_b * T_b


# --------------------------------------------------------------------------
# Growth table, boltzmann.py:177-250, and its interpolation growth.py:7-111.
# --------------------------------------------------------------------------
def growth_integ(cosmo, growth_a, a_lpt_step, rtol=None, atol=None, dt0=1.0):
    eps = np.finfo(np.float64).eps
    tol = math.sqrt(eps)
    rtol = tol if rtol is None else rtol
    atol = tol if atol is None else atol
    a_ic = 0.5 * np.cbrt(eps)
    if a_ic >= a_lpt_step:
        a_ic = 0.1 * a_lpt_step
    a = np.array(growth_a, dtype=np.float64)
    a[0] = a_ic
    lna = np.log(a)

    def ode(G, lna_t):
        at = np.exp(lna_t)
        dlnH = H_deriv(at, cosmo)
        Om = 1.5 * Omega_m_a(at, cosmo)
        G1, G1p, G2, G2p = G[..., 0], G[..., 1], G[..., 2], G[..., 3]
        G1pp = -(3 + dlnH - Om) * G1 - (4 + dlnH) * G1p
        G2pp = Om * G1**2 - (8 + 2 * dlnH - Om) * G2 - (6 + dlnH) * G2p
        return np.stack((G1p, G1pp, G2p, G2pp), axis=-1)

    dtype = np.complex128 if np.iscomplexobj(cosmo.Omega_m) else np.float64
    G_ic = np.array((1, 0, 3 / 7, 0), dtype=dtype)
    G = odeint(ode, G_ic, lna, rtol, atol, dt0=dt0)
    G_deriv = ode(G, lna)
    num_a = len(a)
    G = G.reshape(num_a, 2, 2)
    G_deriv = G_deriv.reshape(num_a, 2, 2)
    G = np.concatenate((G, G_deriv[..., -1:]), axis=2)
    G = np.moveaxis(G, 0, 2)  # (order, deriv, a)
    m = np.array((1, 2), dtype=np.float64)[:, None]
    return np.stack((G[:, 0], m * G[:, 0] + G[:, 1], m**2 * G[:, 0] + 2 * m * G[:, 1] + G[:, 2]), axis=1)


def linear_interp(x, xp, fp):
    """growth.py:7-19 (constant extrapolation)."""
    x = np.asarray(x, dtype=np.float64)
    idx = np.clip(np.searchsorted(xp, x, side='right') - 1, 0, xp.shape[0] - 2)
    x0, x1 = xp[idx], xp[idx + 1]
    y0, y1 = fp[idx], fp[idx + 1]
    y = y0 + (x - x0) * ((y1 - y0) / (x1 - x0))
    y = np.where(x <= xp[0], fp[0], y)
    y = np.where(x >= xp[-1], fp[-1], y)
    return y


def growth(a, cosmo, growth_a, order=1, deriv=0):
    """D_m and its ln-a derivatives, growth.py:75-111."""
    a = np.asarray(a, dtype=np.float64)
    return a**order * linear_interp(a, np.asarray(growth_a, dtype=np.float64), cosmo.growth[order - 1][deriv])


def linear_power(k, a, cosmo, transfer_k, k_pivot_Mpc=0.05, growth_a=None):
    """boltzmann.py:428-484 with the tabulated transfer of boltzmann.py:140-174."""
    k = np.asarray(k, dtype=np.float64)
    T = np.interp(k, transfer_k, cosmo.transfer)
    kp = cosmo.k_pivot(k_pivot_Mpc)
    pw = (k / kp)**cosmo.n_s
    P = 0.32 * cosmo.A_s * kp * pw * (np.pi * (C_LIGHT / H_0)**2 / cosmo.Omega_m * T)**2
    if a is not None:
        P = P * growth(a, cosmo, growth_a)**2
    return P


def tophat_variance(R, cosmo, transfer_k, k_pivot_Mpc=0.05):
    """sigma^2(R) = int dlnk k^3 P(k)/(2 pi^2) W(kR)^2 by Simpson quadrature.

    Restates the quantity of boltzmann.py:292-355 / models.py:249-254; the
    reference evaluates it with mcfit.TophatVar (FFTLog), which is absent, so
    this is a direct quadrature over the transfer table's k range."""
    lnk = np.linspace(np.log(transfer_k[1]), np.log(transfer_k[-1]), 2**16 + 1)
    k = np.exp(lnk)
    P = linear_power(k, None, cosmo, transfer_k, k_pivot_Mpc)
    x = k * R
    W = 3 * (np.sin(x) - x * np.cos(x)) / x**3
    f = k**3 * P / (2 * np.pi**2) * W**2
    h = lnk[1] - lnk[0]
    return h / 3 * (f[0] + f[-1] + 4 * f[1:-1:2].sum() + 2 * f[2:-1:2].sum())


def sigma8(cosmo, transfer_k):
    R = 8 * MPC_SI / UNIT_L
    return math.sqrt(tophat_variance(R, cosmo, transfer_k))
