// Host-side FP64 cosmology: E^2(a), growth ODE (adaptive Dormand-Prince with
// dense output), growth-table interpolation, kick/drift time factors, the
// Eisenstein-Hu transfer fit, the linear power spectrum and the top-hat
// variance.  Everything is templated on the scalar type so Omega_m
// derivatives come from complex-step differentiation (T = std::complex) with
// the step sequence of the real solve.
//
// Reference: cosmology/models.py:16-100 (E2, dlnH/dlna, Omega_m(a)),
// cosmology/boltzmann.py:33-137 (transfer fit), :177-250 (growth ODE),
// :428-484 (linear power), cosmology/growth.py:7-111 (interpolation),
// numerics/ode.py:90-422 (the Dormand-Prince scheme and its step control),
// nbody/integrator.py:114-170 (time factors).
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>

#include "../../include/pmb200.h"

namespace {

using cd = std::complex<double>;
inline double re(double x) { return x; }
inline double re(const cd& x) { return x.real(); }

template <class T>
struct Cos {
  T Om;        // Omega_m
  double Ok;   // Omega_k
  double w0, wa;
  T Ode() const { return 1.0 - (Om + Ok); }
};

template <class T>
T E2(double a, const Cos<T>& c) {
  const double de = std::pow(a, -3 * (1 + c.w0 + c.wa)) * std::exp(-3 * c.wa * (1 - a));
  return c.Om * std::pow(a, -3) + c.Ok * std::pow(a, -2) + c.Ode() * de;
}

template <class T>
T dE2_da(double a, const Cos<T>& c) {
  const double p = -3 * (1 + c.w0 + c.wa), q = -3 * c.wa;
  const double de = std::pow(a, p) * std::exp(q * (1 - a));
  return -3.0 * c.Om * std::pow(a, -4) - 2 * c.Ok * std::pow(a, -3) + c.Ode() * de * (p / a - q);
}

template <class T>
T H_deriv(double a, const Cos<T>& c) {
  return 0.5 * a * dE2_da(a, c) / E2(a, c);
}

template <class T>
T Om_a(double a, const Cos<T>& c) {
  return c.Om / (a * a * a * E2(a, c));
}

template <class T>
void growth_rhs(const T* G, double lna, const Cos<T>& c, T* out) {
  const double a = std::exp(lna);
  const T dlnH = H_deriv(a, c);
  const T Omf = 1.5 * Om_a(a, c);
  out[0] = G[1];
  out[1] = -(3.0 + dlnH - Omf) * G[0] - (4.0 + dlnH) * G[1];
  out[2] = G[3];
  out[3] = Omf * G[0] * G[0] - (8.0 + 2.0 * dlnH - Omf) * G[2] - (6.0 + dlnH) * G[3];
}

// Dormand-Prince tableau (numerics/ode.py:210-221) and dense-output midpoint
// weights (ode.py:108-111).
const double kAlpha[7] = {1 / 5., 3 / 10., 4 / 5., 8 / 9., 1., 1., 0};
const double kBeta[6][7] = {{1 / 5., 0, 0, 0, 0, 0, 0},
                            {3 / 40., 9 / 40., 0, 0, 0, 0, 0},
                            {44 / 45., -56 / 15., 32 / 9., 0, 0, 0, 0},
                            {19372 / 6561., -25360 / 2187., 64448 / 6561., -212 / 729., 0, 0, 0},
                            {9017 / 3168., -355 / 33., 46732 / 5247., 49 / 176., -5103 / 18656., 0, 0},
                            {35 / 384., 0, 500 / 1113., 125 / 192., -2187 / 6784., 11 / 84., 0}};
const double kCsol[7] = {35 / 384., 0, 500 / 1113., 125 / 192., -2187 / 6784., 11 / 84., 0};
const double kCerr[7] = {35 / 384. - 1951 / 21600., 0, 500 / 1113. - 22642 / 50085., 125 / 192. - 451 / 720.,
                         -2187 / 6784. - -12231 / 42400., 11 / 84. - 649 / 6300., -1. / 60.};
const double kCmid[7] = {6025192743. / 30085553152. / 2, 0, 51252292925. / 65400821598. / 2,
                         -2691868925. / 45128329728. / 2, 187940372067. / 1594534317056. / 2,
                         -1776094331. / 19743644256. / 2, 11237099. / 235043384. / 2};

// Integrate the 4-component growth system from ts[0], writing the dense
// solution at every ts[i] (ode.py:351-422: accept if error ratio <= 1, step
// factor min(10, max(0.9 r^-1/5, 0.2 or 1)), quartic interpolation).
template <class T>
void odeint_growth(const Cos<T>& c, const std::vector<double>& ts, double rtol, double atol, double dt0,
                   std::vector<T>& out) {
  const int D = 4;
  out.assign(ts.size() * D, T(0));
  T y[D] = {T(1), T(0), T(3.0 / 7.0), T(0)};
  T f[D];
  growth_rhs(y, ts[0], c, f);
  double t = ts[0], last_t = t, dt = dt0;
  T coeff[5][D];
  for (int j = 0; j < 5; ++j)
    for (int d = 0; d < D; ++d) coeff[j][d] = y[d];
  for (int d = 0; d < D; ++d) out[d] = y[d];
  for (size_t it = 1; it < ts.size(); ++it) {
    const double target = ts[it];
    while (t < target && dt > 0) {
      T k[7][D];
      for (int d = 0; d < D; ++d) k[0][d] = f[d];
      for (int i = 1; i < 7; ++i) {
        T yi[D];
        for (int d = 0; d < D; ++d) {
          T s = 0;
          for (int j = 0; j < 7; ++j) s += kBeta[i - 1][j] * k[j][d];
          yi[d] = y[d] + dt * s;
        }
        growth_rhs(yi, t + dt * kAlpha[i - 1], c, k[i]);
      }
      T ny[D], err[D], ymid[D];
      for (int d = 0; d < D; ++d) {
        T s = 0, e = 0, mm = 0;
        for (int j = 0; j < 7; ++j) {
          s += kCsol[j] * k[j][d];
          e += kCerr[j] * k[j][d];
          mm += kCmid[j] * k[j][d];
        }
        ny[d] = dt * s + y[d];
        err[d] = dt * e;
        ymid[d] = y[d] + dt * mm;
      }
      double ms = 0;
      for (int d = 0; d < D; ++d) {
        const double tol = atol + rtol * std::max(std::fabs(re(y[d])), std::fabs(re(ny[d])));
        const double r = re(err[d]) / tol;
        ms += r * r;
      }
      const double ratio = std::sqrt(ms / D);
      double ndt;
      if (ratio == 0) {
        ndt = dt * 10.0;
      } else {
        const double dfac = ratio < 1 ? 1.0 : 0.2;
        ndt = dt * std::min(10.0, std::max(std::pow(ratio, -1.0 / 5.0) * 0.9, dfac));
      }
      if (ndt < 0) ndt = 0;
      if (ratio <= 1.0) {
        for (int d = 0; d < D; ++d) {
          const T dy0 = k[0][d], dy1 = k[6][d];
          coeff[0][d] = -2. * dt * dy0 + 2. * dt * dy1 - 8. * y[d] - 8. * ny[d] + 16. * ymid[d];
          coeff[1][d] = 5. * dt * dy0 - 3. * dt * dy1 + 18. * y[d] + 14. * ny[d] - 32. * ymid[d];
          coeff[2][d] = -4. * dt * dy0 + dt * dy1 - 11. * y[d] - 5. * ny[d] + 16. * ymid[d];
          coeff[3][d] = dt * dy0;
          coeff[4][d] = y[d];
          y[d] = ny[d];
          f[d] = k[6][d];
        }
        last_t = t;
        t = t + dt;
      }
      dt = ndt;
    }
    const double x = (target - last_t) / (t - last_t);
    for (int d = 0; d < D; ++d) {
      T v = coeff[0][d];
      for (int j = 1; j < 5; ++j) v = v * x + coeff[j][d];
      out[it * D + d] = v;
    }
  }
}

// growth table [order(2)][deriv(3)][na] (boltzmann.py:236-249)
template <class T>
void growth_table(const Cos<T>& c, const double* growth_a, int na, double a_lpt_step, double rtol, double atol,
                  double dt0, std::vector<T>& table) {
  const double eps = 2.220446049250313e-16;
  double a_ic = 0.5 * std::cbrt(eps);
  if (a_ic >= a_lpt_step) a_ic = 0.1 * a_lpt_step;
  std::vector<double> lna(na);
  for (int i = 0; i < na; ++i) lna[i] = std::log(i == 0 ? a_ic : growth_a[i]);
  std::vector<T> G;
  odeint_growth(c, lna, rtol, atol, dt0, G);
  table.assign(6 * (size_t)na, T(0));
  for (int i = 0; i < na; ++i) {
    T g[4], gd[4];
    for (int d = 0; d < 4; ++d) g[d] = G[(size_t)i * 4 + d];
    growth_rhs(g, lna[i], c, gd);
    for (int m = 1; m <= 2; ++m) {
      const T G0 = g[2 * (m - 1)], G1 = g[2 * (m - 1) + 1], G2 = gd[2 * (m - 1) + 1];
      const double mm = m;
      table[((m - 1) * 3 + 0) * (size_t)na + i] = G0;
      table[((m - 1) * 3 + 1) * (size_t)na + i] = mm * G0 + G1;
      table[((m - 1) * 3 + 2) * (size_t)na + i] = mm * mm * G0 + 2 * mm * G1 + G2;
    }
  }
}

// growth.py:7-19 (constant extrapolation), times a^order (growth.py:109)
template <class T>
T growth_at(double a, const double* ga, int na, const T* tab, int order, int deriv) {
  const T* fp = tab + ((order - 1) * 3 + deriv) * (size_t)na;
  T y;
  if (a <= ga[0]) {
    y = fp[0];
  } else if (a >= ga[na - 1]) {
    y = fp[na - 1];
  } else {
    int lo = 0, hi = na;  // searchsorted right - 1
    while (lo < hi) {
      int mid = (lo + hi) / 2;
      if (ga[mid] <= a) lo = mid + 1; else hi = mid;
    }
    int idx = lo - 1;
    if (idx < 0) idx = 0;
    if (idx > na - 2) idx = na - 2;
    y = fp[idx] + (a - ga[idx]) * ((fp[idx + 1] - fp[idx]) / (ga[idx + 1] - ga[idx]));
  }
  return std::pow(a, (double)order) * y;
}

template <class T>
T G_D(double a, const Cos<T>& c, const double* ga, int na, const T* tab) {
  return a * a * std::sqrt(E2(a, c)) * growth_at(a, ga, na, tab, 1, 1);
}

template <class T>
T G_K(double a, const Cos<T>& c, const double* ga, int na, const T* tab) {
  return a * a * a * E2(a, c) *
         (growth_at(a, ga, na, tab, 1, 2) + (2.0 + H_deriv(a, c)) * growth_at(a, ga, na, tab, 1, 1));
}

}  // namespace

extern "C" {

int pmb_growth_table(double omega_m, double omega_k, double w0, double wa, const double* growth_a, int na,
                     double a_lpt_step, double rtol, double atol, double dt0, double* table, double* dtable_dom) {
  if (na < 2 || growth_a == nullptr || table == nullptr) return -1;
  Cos<double> c{omega_m, omega_k, w0, wa};
  std::vector<double> t;
  growth_table(c, growth_a, na, a_lpt_step, rtol, atol, dt0, t);
  std::memcpy(table, t.data(), sizeof(double) * t.size());
  if (dtable_dom != nullptr) {
    const double h = 1e-30;
    Cos<cd> cc{cd(omega_m, h), omega_k, w0, wa};
    std::vector<cd> tc;
    growth_table(cc, growth_a, na, a_lpt_step, rtol, atol, dt0, tc);
    for (size_t i = 0; i < tc.size(); ++i) dtable_dom[i] = tc[i].imag() / h;
  }
  return 0;
}

// Kick/drift factors of one macro step (integrator.py:125-170) and their
// derivatives w.r.t. Omega_m.  kind 0: drift(a_vel=a0, a_prev=a1, a_next=a2);
// kind 1: kick(a_acc=a0, a_prev=a1, a_next=a2).
int pmb_time_factor(int kind, double a0, double a1, double a2, double omega_m, double omega_k, double w0, double wa,
                    const double* growth_a, int na, const double* table, const double* dtable_dom, double* factor,
                    double* dfactor_dom) {
  if (na < 2 || factor == nullptr) return -1;
  Cos<double> c{omega_m, omega_k, w0, wa};
  if (kind == 0) {
    *factor = (growth_at(a2, growth_a, na, table, 1, 0) - growth_at(a1, growth_a, na, table, 1, 0)) /
              G_D(a0, c, growth_a, na, table);
  } else {
    *factor = (G_D(a2, c, growth_a, na, table) - G_D(a1, c, growth_a, na, table)) / G_K(a0, c, growth_a, na, table);
  }
  if (dfactor_dom != nullptr && dtable_dom != nullptr) {
    const double h = 1e-30;
    Cos<cd> cc{cd(omega_m, h), omega_k, w0, wa};
    std::vector<cd> tab((size_t)6 * na);
    for (size_t i = 0; i < tab.size(); ++i) tab[i] = cd(table[i], h * dtable_dom[i]);
    cd f;
    if (kind == 0) {
      f = (growth_at(a2, growth_a, na, tab.data(), 1, 0) - growth_at(a1, growth_a, na, tab.data(), 1, 0)) /
          G_D(a0, cc, growth_a, na, tab.data());
    } else {
      f = (G_D(a2, cc, growth_a, na, tab.data()) - G_D(a1, cc, growth_a, na, tab.data())) /
          G_K(a0, cc, growth_a, na, tab.data());
    }
    *dfactor_dom = f.imag() / h;
  }
  return 0;
}

// D_m(a), dD_m/dlna(a) and a^2 H dD_m/dlna for LPT (lpt.py:412-417) with
// Omega_m derivatives: out[order-1][0..2], dout likewise.
int pmb_lpt_factors(double a, double omega_m, double omega_k, double w0, double wa, const double* growth_a, int na,
                    const double* table, const double* dtable_dom, double* out, double* dout) {
  if (na < 2 || out == nullptr) return -1;
  Cos<double> c{omega_m, omega_k, w0, wa};
  for (int m = 1; m <= 2; ++m) {
    const double D = growth_at(a, growth_a, na, table, m, 0);
    const double dD = growth_at(a, growth_a, na, table, m, 1);
    out[(m - 1) * 3 + 0] = D;
    out[(m - 1) * 3 + 1] = dD;
    out[(m - 1) * 3 + 2] = a * a * std::sqrt(E2(a, c)) * dD;
  }
  if (dout != nullptr && dtable_dom != nullptr) {
    const double h = 1e-30;
    Cos<cd> cc{cd(omega_m, h), omega_k, w0, wa};
    std::vector<cd> tab((size_t)6 * na);
    for (size_t i = 0; i < tab.size(); ++i) tab[i] = cd(table[i], h * dtable_dom[i]);
    for (int m = 1; m <= 2; ++m) {
      const cd D = growth_at(a, growth_a, na, tab.data(), m, 0);
      const cd dD = growth_at(a, growth_a, na, tab.data(), m, 1);
      dout[(m - 1) * 3 + 0] = D.imag() / h;
      dout[(m - 1) * 3 + 1] = dD.imag() / h;
      dout[(m - 1) * 3 + 2] = (a * a * std::sqrt(E2(a, cc)) * dD).imag() / h;
    }
  }
  return 0;
}

// Eisenstein & Hu transfer fit (boltzmann.py:33-137) at k [1/L] (h/Mpc units).
int pmb_transfer_fit(const double* k, int64_t nk, double omega_m, double omega_b, double h, double T_cmb,
                     int nowiggle, double* out) {
  if (k == nullptr || out == nullptr) return -1;
  const double T2 = (T_cmb / 2.7) * (T_cmb / 2.7);
  const double h2 = h * h, w_m = omega_m * h2, w_b = omega_b * h2;
  const bool zero_b = w_b <= 0;
  const double w_b_safe = zero_b ? 1e-8 : w_b;
  const double f_b = omega_b / omega_m, f_c = (omega_m - omega_b) / omega_m;
  const double z_eq = 2.50e4 * w_m / (T2 * T2), k_eq = 7.46e-2 * w_m / T2;
  double b1 = 0.313 * std::pow(w_m, -0.419) * (1 + 0.607 * std::pow(w_m, 0.674));
  double b2 = 0.238 * std::pow(w_m, 0.223);
  const double z_d = 1291 * std::pow(w_m, 0.251) / (1 + 0.659 * std::pow(w_m, 0.828)) * (1 + b1 * std::pow(w_b, b2));
  const double R_d = 31.5 * w_b_safe / (T2 * T2) * (1e3 / z_d);
  const double R_eq = 31.5 * w_b_safe / (T2 * T2) * (1e3 / z_eq);
  const double s = 2 / (3 * k_eq) * std::sqrt(6 / R_eq) *
                   std::log((std::sqrt(1 + R_d) + std::sqrt(R_eq + R_d)) / (1 + std::sqrt(R_eq)));
  const double k_silk = 1.6 * std::pow(w_b, 0.52) * std::pow(w_m, 0.73) * (1 + std::pow(10.4 * w_m, -0.95));
  const double a1 = std::pow(46.9 * w_m, 0.670) * (1 + std::pow(32.1 * w_m, -0.532));
  const double a2 = std::pow(12.0 * w_m, 0.424) * (1 + std::pow(45.0 * w_m, -0.582));
  const double alpha_c = std::pow(a1, -f_b) * std::pow(a2, -f_b * f_b * f_b);
  b1 = 0.944 / (1 + std::pow(458 * w_m, -0.708));
  b2 = std::pow(0.395 * w_m, -0.0266);
  const double beta_c = 1 / (1 + b1 * (std::pow(f_c, b2) - 1));
  const double y = (1 + z_eq) / (1 + z_d), x = std::sqrt(1 + y);
  const double G = y * (-6 * x + (2 + 3 * y) * std::log((x + 1) / (x - 1)));
  const double alpha_b = 2.07 * k_eq * s * std::pow(1 + R_d, -0.75) * G;
  const double beta_node = 8.41 * std::pow(w_m, 0.435);
  const double beta_b = 0.5 + f_b + (3 - 2 * f_b) * std::sqrt(1 + (17.2 * w_m) * (17.2 * w_m));
  auto T0 = [&](double kk, double ac, double bc) {
    const double q = kk / (13.41 * k_eq);
    const double L = std::log(M_E + 1.8 * bc * q);
    const double C = 14.2 / ac + 386 / (1 + 69.9 * std::pow(q, 1.08));
    return L / (L + C * q * q);
  };
  for (int64_t i = 0; i < nk; ++i) {
    const double kk = k[i] * h;  // k * h / L * Mpc_SI with L = Mpc_SI
    if (nowiggle) {
      const double ag = 1 - 0.328 * std::log(431 * w_m) * f_b + 0.38 * std::log(22.3 * w_m) * f_b * f_b;
      const double ger = ag + (1 - ag) / (1 + std::pow(0.43 * kk * s, 4));
      const double qe = kk / (13.41 * k_eq * ger);
      const double L0 = std::log(2 * M_E + 1.8 * qe), C0 = 14.2 + 731 / (1 + 62.5 * qe);
      out[i] = L0 / (L0 + C0 * qe * qe);
      continue;
    }
    const double tnb = T0(kk, 1, 1);
    if (zero_b) {
      out[i] = tnb;
      continue;
    }
    const double f = 1 / (1 + std::pow(kk * s / 5.4, 4));
    const double Tc = f * T0(kk, 1, beta_c) + (1 - f) * T0(kk, alpha_c, beta_c);
    const double ks = kk * s;
    const double arg = ks * ks / (M_PI * std::cbrt(beta_node * beta_node * beta_node + ks * ks * ks));
    const double sinc = arg == 0 ? 1.0 : std::sin(M_PI * arg) / (M_PI * arg);
    const double Tb = (tnb / (1 + (ks / 5.2) * (ks / 5.2)) +
                       alpha_b * ks * ks * ks / (beta_b * beta_b * beta_b + ks * ks * ks) *
                           std::exp(-std::pow(kk / k_silk, 1.4))) * sinc;
    out[i] = f_c * Tc + f_b * Tb;
  }
  return 0;
}

// Linear power (boltzmann.py:428-484) from a tabulated transfer (linear
// interpolation with constant extrapolation, boltzmann.py:170), no growth.
int pmb_linear_power(const double* k, int64_t nk, const double* tk, const double* tt, int ntab, double A_s,
                     double n_s, double omega_m, double h, double k_pivot_Mpc, double* out) {
  if (k == nullptr || tk == nullptr || tt == nullptr || out == nullptr || ntab < 2) return -1;
  const double c_light = 299792458.0 / 1e5;  // c_SI / V with V = 1e5 m/s
  const double kp = k_pivot_Mpc / h;
  for (int64_t i = 0; i < nk; ++i) {
    const double kk = k[i];
    double T;
    if (kk <= tk[0]) {
      T = tt[0];
    } else if (kk >= tk[ntab - 1]) {
      T = tt[ntab - 1];
    } else {
      int lo = 0, hi = ntab - 1;
      while (hi - lo > 1) {
        int mid = (lo + hi) / 2;
        if (tk[mid] <= kk) lo = mid; else hi = mid;
      }
      T = tt[lo] + (kk - tk[lo]) * (tt[hi] - tt[lo]) / (tk[hi] - tk[lo]);
    }
    const double amp = M_PI * c_light * c_light / omega_m * T;
    out[i] = 0.32 * A_s * kp * std::pow(kk / kp, n_s) * amp * amp;
  }
  return 0;
}

}  // extern "C"
