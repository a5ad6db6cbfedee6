// Jacobi-Davidson corrections for the mixed form of the device Davidson.
//
// The reference's Davidson expands its basis with t = -P r, P the bounded
// kinetic preconditioner (src/pw_core.cpp:1384-1401). The mixed form replaces
// that single preconditioner step by a few steps of preconditioned conjugate
// gradients on the Jacobi-Davidson correction equation of every unconverged
// root c (Ritz pair x_c, theta_c, residual r_c):
//
//   (I - S X X^H) (H - theta_c S) (I - X X^H S) t_c = -r_c,   X^H S t_c = 0,
//
// X the block of Ritz vectors. On the S-orthogonal complement of X the
// shifted operator is positive for the lowest roots, so CG applies; P (with
// the Ritz vector's kinetic energy) preconditions it. The operator is applied
// in the mixed form (FP32 FFT, BF16-split PAW products) and the projections
// run on the tensor cores: the corrections only steer the search, while the
// basis, the Galerkin pencil, the Rayleigh-Ritz step and the certificate keep
// their own precision. Far fewer outer iterations (each with an FP64
// Rayleigh-Ritz) follow than with the single preconditioner step.
#pragma once

#include "operator.cuh"
#include "umma_gemm.cuh"

namespace sdft_b200 {

// out (n x count, ld n) <- the corrections of the roots selected[0..count)
// after `steps` CG steps. x, sx: n x roots Ritz vectors and their S images
// (S-orthonormal), r: n x roots residuals, theta: device Ritz values (roots),
// selected: host root indices. All device arrays on the operator's stream.
void jacobi_davidson_corrections(DeviceOperator& op, CorrectionBuffers& buf, const Cx<double>* x,
                                 const Cx<double>* sx, const Cx<double>* r, const double* theta, int roots,
                                 const int* selected, int count, int steps, Cx<double>* out);

}  // namespace sdft_b200
