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

}  // namespace pbe
}  // namespace sdft_b200
