// Spin-unpolarised PBE exchange-correlation of one grid point in FP64 (the
// reference's pbe_unpolarized, src/pbe_xc.cpp:75-140, and its CUDA port
// src/cuda_pbe.cuh:22-55), shared by the per-point kernel and the fused XC
// functional. Forward-mode duals carry d/dn and d/d|grad n|^2 through PBE
// exchange (Perdew, Burke & Ernzerhof, PRL 77, 3865 (1996)) and PW92
// correlation (Perdew & Wang, PRB 45, 13244 (1992)); the sigma response uses
// the cancellation-free difference of the two enhancement factors.
#pragma once

#include "common.cuh"

namespace sdft_b200 {
namespace pbe {

// Physical constants of the PBE and PW92 functionals (the published values,
// identical to the reference so that results agree to rounding).
inline constexpr double kPi = 3.1415926535897932384626433832795;
inline constexpr double kGamma = 0.031090690869654895;  // (1 - ln 2)/pi^2
inline constexpr double kBeta = 0.06672455060314922;
inline constexpr double kMu = 0.2195149727645171;       // beta pi^2 / 3
inline constexpr double kKappa = 0.804;
inline constexpr double kPwA = 0.0310907, kPwAlpha1 = 0.21370, kPwB1 = 7.5957, kPwB2 = 3.5876, kPwB3 = 1.6382,
                 kPwB4 = 0.49294;

struct Dual {
  double v, dn, dg;  // value, d/dn, d/d(|grad n|^2)
};
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.dn + b.dn, a.dg + b.dg}; }
__device__ __forceinline__ Dual operator-(Dual a) { return {-a.v, -a.dn, -a.dg}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) {
  return {a.v * b.v, a.dn * b.v + a.v * b.dn, a.dg * b.v + a.v * b.dg};
}
__device__ __forceinline__ Dual operator/(Dual a, Dual b) {
  const double inv = 1.0 / b.v, inv2 = inv * inv;
  return {a.v * inv, (a.dn * b.v - a.v * b.dn) * inv2, (a.dg * b.v - a.v * b.dg) * inv2};
}
__device__ __forceinline__ Dual operator+(double a, Dual b) { return {a + b.v, b.dn, b.dg}; }
__device__ __forceinline__ Dual operator-(double a, Dual b) { return {a - b.v, -b.dn, -b.dg}; }
__device__ __forceinline__ Dual operator*(Dual a, double b) { return {a.v * b, a.dn * b, a.dg * b}; }
__device__ __forceinline__ Dual operator*(double a, Dual b) { return {a * b.v, a * b.dn, a * b.dg}; }
__device__ __forceinline__ Dual operator/(double a, Dual b) { return Dual{a, 0.0, 0.0} / b; }
__device__ __forceinline__ Dual operator/(Dual a, double b) { return a * (1.0 / b); }

__device__ __forceinline__ Dual dpow(Dual x, double p) {
  const double value = p == 0.5 ? sqrt(x.v) : pow(x.v, p);
  const double d = p * value / x.v;
  return {value, d * x.dn, d * x.dg};
}
__device__ __forceinline__ Dual dlog1p(Dual x) { return {log1p(x.v), x.dn / (1.0 + x.v), x.dg / (1.0 + x.v)}; }
__device__ __forceinline__ Dual dexpm1(Dual x) {
  const double value = expm1(x.v);
  return {value, (1.0 + value) * x.dn, (1.0 + value) * x.dg};
}

__device__ __forceinline__ Dual pw92(Dual rs) {
  const Dual root = dpow(rs, 0.5);
  const Dual poly = kPwB1 * root + kPwB2 * rs + kPwB3 * rs * root + kPwB4 * rs * rs;
  return -2.0 * kPwA * (1.0 + kPwAlpha1 * rs) * dlog1p(1.0 / (2.0 * kPwA * poly));
}

struct Point {
  double energy, exchange_energy, correlation_energy, vx, vc, sigma;
};

__device__ __forceinline__ Point pbe_point(double density, double gradient_magnitude) {
  const Dual n{density, 1.0, 0.0};
  const Dual g2{gradient_magnitude * gradient_magnitude, 0.0, 1.0};
  const Dual root_n = dpow(n, 1.0 / 3.0);
  const Dual rs = cbrt(3.0 / (4.0 * kPi)) / root_n;
  const Dual kf = cbrt(3.0 * kPi * kPi) * root_n;
  const Dual eps_x = (-0.75 * cbrt(3.0 / kPi)) * root_n;
  const Dual s2 = g2 / (4.0 * kf * kf * n * n);
  const Dual fx = 1.0 + kKappa - kKappa / (1.0 + (kMu / kKappa) * s2);
  const Dual exchange = n * eps_x * fx;
  const Dual eps_c = pw92(rs);
  const Dual ks2 = 4.0 * kf / kPi;
  const Dual t2 = g2 / (4.0 * ks2 * n * n);
  const Dual em1 = dexpm1(-eps_c / kGamma);
  const Dual a = (kBeta / kGamma) / em1;
  const Dual at2 = a * t2;
  const Dual t4a2 = at2 * at2;
  const Dual h = kGamma * dlog1p((kBeta / kGamma) * t2 * (1.0 + at2) / (1.0 + at2 + t4a2));
  const Dual correlation = n * (eps_c + h);
  // Cancellation-free sigma response (mu = beta pi^2/3 makes the exchange and
  // correlation derivatives cancel at sigma = 0).
  const double u = (kMu / kKappa) * s2.v, x = at2.v, den = 1.0 + x + x * x;
  const double bt = (kBeta / kGamma) * t2.v * (1.0 + x);
  double difference;
  if (u > 0.25 || x > 0.25) {
    difference = (1.0 + 2.0 * x) / (den * (den + bt)) - 1.0 / ((1.0 + u) * (1.0 + u));
  } else {
    const double exchange_loss = u * (2.0 + u) / ((1.0 + u) * (1.0 + u));
    const double correlation_loss = (x * x * (3.0 + x * (2.0 + x)) + bt * den) / (den * (den + bt));
    difference = exchange_loss - correlation_loss;
  }
  Point p;
  p.exchange_energy = exchange.v;
  p.correlation_energy = correlation.v;
  p.energy = exchange.v + correlation.v;
  p.vx = exchange.dn;
  p.vc = correlation.dn;
  p.sigma = kBeta / (2.0 * ks2.v * n.v) * difference;
  return p;
}

// ---- Collinear (spin) PBE with PW92 spin interpolation ---------------------
// The reference's pbe_collinear (src/spin_pbe_xc.cpp:54-107): forward
// derivatives in five independent variables (n_up, n_down, sigma_uu,
// sigma_ud, sigma_dd), exchange by spin scaling with the bounded enhancement
// form, correlation with the PW92 f(zeta) interpolation and the regularised
// phi derivative (eta = 1e-12), zeta clamped to +-(1 - 1e-13) in value only.
struct D5 {
  double v, g[5];
};
__device__ __forceinline__ D5 d5(double x) { return {x, {0, 0, 0, 0, 0}}; }
__device__ __forceinline__ D5 d5_variable(double x, int k) {
  D5 r = d5(x);
  r.g[k] = 1.0;
  return r;
}
__device__ __forceinline__ D5 operator+(D5 a, D5 b) {
  D5 r{a.v + b.v, {}};
  for (int i = 0; i < 5; ++i) r.g[i] = a.g[i] + b.g[i];
  return r;
}
__device__ __forceinline__ D5 operator-(D5 a, D5 b) {
  D5 r{a.v - b.v, {}};
  for (int i = 0; i < 5; ++i) r.g[i] = a.g[i] - b.g[i];
  return r;
}
__device__ __forceinline__ D5 operator-(D5 a) { return d5(0.0) - a; }
__device__ __forceinline__ D5 operator*(D5 a, D5 b) {
  D5 r{a.v * b.v, {}};
  for (int i = 0; i < 5; ++i) r.g[i] = a.g[i] * b.v + a.v * b.g[i];
  return r;
}
__device__ __forceinline__ D5 operator/(D5 a, D5 b) {
  D5 r{a.v / b.v, {}};
  for (int i = 0; i < 5; ++i) r.g[i] = (a.g[i] - r.v * b.g[i]) / b.v;
  return r;
}
__device__ __forceinline__ D5 operator+(double a, D5 b) { return d5(a) + b; }
__device__ __forceinline__ D5 operator-(double a, D5 b) { return d5(a) - b; }
__device__ __forceinline__ D5 operator*(double a, D5 b) { return d5(a) * b; }
__device__ __forceinline__ D5 operator/(double a, D5 b) { return d5(a) / b; }
__device__ __forceinline__ D5 operator+(D5 a, double b) { return a + d5(b); }
__device__ __forceinline__ D5 operator-(D5 a, double b) { return a - d5(b); }
__device__ __forceinline__ D5 operator*(D5 a, double b) { return a * d5(b); }
__device__ __forceinline__ D5 operator/(D5 a, double b) { return a / d5(b); }
__device__ __forceinline__ D5 d5_pow(D5 a, double p) {
  D5 r{pow(a.v, p), {}};
  for (int i = 0; i < 5; ++i) r.g[i] = p * r.v / a.v * a.g[i];
  return r;
}
__device__ __forceinline__ D5 d5_log1p(D5 a) {
  D5 r{log1p(a.v), {}};
  for (int i = 0; i < 5; ++i) r.g[i] = a.g[i] / (1 + a.v);
  return r;
}
__device__ __forceinline__ D5 d5_expm1(D5 a) {
  D5 r{expm1(a.v), {}};
  for (int i = 0; i < 5; ++i) r.g[i] = (1 + r.v) * a.g[i];
  return r;
}
// PW92 G(rs; A, alpha1, beta1..beta4).
__device__ __forceinline__ D5 pw92_spin(D5 r, double a, double alpha, double b1, double b2, double b3, double b4) {
  const D5 root = d5_pow(r, .5);
  const D5 poly = b1 * root + b2 * r + b3 * r * root + b4 * r * r;
  return -2 * a * (1 + alpha * r) * d5_log1p(1 / (2 * a * poly));
}
// Spin-scaled exchange .5 E_x[2 n_s, 2 grad n_s] with the bounded enhancement.
__device__ __forceinline__ D5 spin_exchange(D5 n, D5 sigma) {
  const D5 doubled = 2 * n;
  const D5 root = d5_pow(doubled, 1. / 3.);
  const D5 kf = cbrt(3 * kPi * kPi) * root;
  const D5 denominator = 4 * kf * kf * doubled * doubled;
  const D5 numerator = 4 * (kMu / kKappa) * sigma;
  const D5 fx = 1 + kKappa * numerator / (denominator + numerator);
  return -.375 * cbrt(3 / kPi) * doubled * root * fx;
}

struct SpinPoint {
  double energy, density_potential[2], gradient_response[2][3];
};

// up, down > 0 (the caller's floors); gu, gd the channel gradients.
__device__ __forceinline__ SpinPoint pbe_collinear(double up, double down, const double gu[3], const double gd[3]) {
  double uu = 0, ud = 0, dd = 0;
  for (int a = 0; a < 3; ++a) {
    uu += gu[a] * gu[a];
    ud += gu[a] * gd[a];
    dd += gd[a] * gd[a];
  }
  const D5 nu = d5_variable(fmax(up, 1e-99), 0), nd = d5_variable(fmax(down, 1e-99), 1);
  const D5 su = d5_variable(uu, 2), sud = d5_variable(ud, 3), sd = d5_variable(dd, 4);
  const D5 n = nu + nd, root = d5_pow(n, 1. / 3.), rs = cbrt(3 / (4 * kPi)) / root;
  D5 z = (nu - nd) / n;
  z.v = fmin(fmax(z.v, -.9999999999999), .9999999999999);
  const D5 z2 = z * z, z4 = z2 * z2;
  const D5 pu = 1 + z, pd = 1 - z;
  constexpr double denominator = 0.5198420997897463295;
  constexpr double fzz = 8 / (9 * denominator);
  const D5 f = (d5_pow(pu, 4. / 3.) + d5_pow(pd, 4. / 3.) - 2) / denominator;
  const D5 eu = pw92_spin(rs, .0310907, .21370, 7.5957, 3.5876, 1.6382, .49294);
  const D5 ep = pw92_spin(rs, .01554535, .20548, 14.1189, 6.1977, 3.3662, .62517);
  const D5 alpha = -pw92_spin(rs, .0168869, .11125, 10.357, 3.6231, .88026, .49671);
  const D5 ec = eu + alpha * f / fzz * (1 - z4) + (ep - eu) * f * z4;
  D5 phi = .5 * (d5_pow(pu, 2. / 3.) + d5_pow(pd, 2. / 3.));
  constexpr double eta = 1e-12;
  const double gz = (pow(pu.v * pu.v + eta, -1. / 6.) - pow(pd.v * pd.v + eta, -1. / 6.)) / 3.;
  for (int i = 0; i < 5; ++i) phi.g[i] = gz * z.g[i];
  const D5 phi3 = phi * phi * phi;
  const D5 sigma = su + 2 * sud + sd;
  const D5 kf = cbrt(3 * kPi * kPi) * root, ks2 = 4 * kf / kPi;
  const D5 t2 = sigma / (4 * phi * phi * ks2 * n * n);
  const D5 a = (kBeta / kGamma) / d5_expm1(-ec / (kGamma * phi3));
  const D5 at = a * t2;
  const D5 h = kGamma * phi3 * d5_log1p((kBeta / kGamma) * t2 * (1 + at) / (1 + at + at * at));
  D5 ex = up == 0 ? d5(0.0) : spin_exchange(nu, su);
  if (down != 0) ex = ex + spin_exchange(nd, sd);
  const D5 co = n * (ec + h), total = ex + co;
  SpinPoint out;
  out.energy = total.v;
  out.density_potential[0] = total.g[0];
  out.density_potential[1] = total.g[1];
  for (int axis = 0; axis < 3; ++axis) {
    out.gradient_response[0][axis] = 2 * total.g[2] * gu[axis] + total.g[3] * gd[axis];
    out.gradient_response[1][axis] = 2 * total.g[4] * gd[axis] + total.g[3] * gu[axis];
  }
  return out;
}

}  // namespace pbe
}  // namespace sdft_b200
