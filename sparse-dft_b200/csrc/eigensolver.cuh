// Lowest eigenpairs of a small dense Hermitian matrix on the device, for the
// Davidson Rayleigh-Ritz step: one cooperative kernel reduces the matrix to
// real symmetric tridiagonal form (Householder, LAPACK zhetd2 conventions),
// multisection on Sturm counts gives the wanted eigenvalues, inverse
// iteration (with Gram-Schmidt inside tight clusters) their tridiagonal
// eigenvectors, and the Householder reflectors are applied back.
#pragma once
#include <cublas_v2.h>
#include <cusolverDn.h>

#include "common.cuh"
#include "gemm.cuh"

namespace sdft_b200 {

struct EigenWorkspace {
  Scratch tridiagonal;  // d, e, tau, reflectors, exchange buffers, barrier words
  Scratch vectors;      // tridiagonal eigenvectors and inverse-iteration factors
  Scratch scalar;       // reduction word
  Scratch product;      // m x m products for the overlap correction
  Scratch product2;
  Scratch solver_work;  // cuSOLVER workspace and info word (generalized fallback)
};

enum class RitzSolver : int { Device = 0, Subset = 1, Full = 2 };

// SDFT_B200_RR: device (default), subset (cuSOLVER zhegvdx) or full (zhegvd).
RitzSolver rr_mode();

// Largest matrix order the tridiagonalization kernel holds in shared memory.
int hermitian_eigen_max_order();

// a: m x m Hermitian (both triangles), column-major with leading dimension
// m; overwritten. On return values[0..wanted) (device) holds the lowest
// eigenvalues in ascending order and vectors (m x wanted, leading dimension
// m, device; may alias a) the orthonormal eigenvectors. m must not exceed
// hermitian_eigen_max_order(). blas must be bound to `stream`.
void hermitian_lowest(cublasHandle_t blas, Cx<double>* a, int m, int wanted, double* values, Cx<double>* vectors,
                      EigenWorkspace& ws, cudaStream_t stream);

// Lowest `wanted` pairs of the Hermitian pencil H y = e S y (the reference's
// rayleigh_ritz, src/pw_core.cpp:56-136). h, s: m x m, both triangles,
// leading dimension m, device; both overwritten. values: device, at least
// `wanted` (all m for RitzSolver::Full); vectors: m x wanted (m x m for
// Full), leading dimension m, may alias h, S-orthonormal.
// Device solver on S = I + E: nothing when max |E| <= 1e-14; the
// first-order Loewdin transform C = I - E/2 (H' = H - (E H + H E)/2,
// y -> y - E y/2, error O(|E|^2)) up to first_order_limit; the second-order
// C = I - E/2 + 3/8 E^2 (H' = C H C, y -> C y, error O(|E|^3)) up to
// max_deviation.
// Beyond that, or when m exceeds hermitian_eigen_max_order(), cuSOLVER
// zhegvdx solves the pencil.
void generalized_lowest(cublasHandle_t blas, cusolverDnHandle_t solver, Cx<double>* h, Cx<double>* s, int m,
                        int wanted, double* values, Cx<double>* vectors, EigenWorkspace& ws, RitzSolver mode,
                        cudaStream_t stream, double max_deviation = 1e-5, double first_order_limit = 1e-8);

// b <- b - I (m x m, leading dimension m); returns max |entry| of the result.
double identity_deviation(Cx<double>* b, int m, EigenWorkspace& ws, cudaStream_t stream);

// b <- b + I (m x m, leading dimension m).
void add_identity(Cx<double>* b, int m, cudaStream_t stream);

// a <- a - (f + f^H) / 2 (m x m, leading dimension m).
void lowdin_combine(Cx<double>* a, const Cx<double>* f, int m, cudaStream_t stream);

}  // namespace sdft_b200
