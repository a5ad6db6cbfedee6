// The reference's bounded rational kinetic preconditioner
// (src/pw_core.cpp:33-47), shared by the Davidson kernels.
#pragma once

namespace sdft_b200 {

// 2/s * p(x) / (p(x) + 16 x^4) with x = T / s, s = 1.5 max(<T>_psi, 2/27.211386245988),
// evaluated in the reference's two branches.
__device__ __forceinline__ double kinetic_preconditioner(double kinetic, double wavefunction_kinetic) {
  const double scale = 1.5 * fmax(wavefunction_kinetic, 2.0 / 27.211386245988);
  const double x = kinetic / scale;
  if (x > 1.0) {
    const double inv = 1.0 / x;
    const double p = inv * (8.0 + inv * (12.0 + inv * (18.0 + 27.0 * inv)));
    return (2.0 / scale) * p / (p + 16.0);
  }
  const double p = 27.0 + x * (18.0 + x * (12.0 + 8.0 * x));
  return (2.0 / scale) * p / (p + 16.0 * x * x * x * x);
}

}  // namespace sdft_b200
