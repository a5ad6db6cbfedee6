// Column-wise reductions and small dense helpers for the device Davidson solver.
#pragma once
#include "common.cuh"

namespace sdft_b200 {

// dst(m x m, ldd) = (src + src^H)/2.
void hermitian_part(const Cx<double>* src, long long lds, Cx<double>* dst, long long ldd, int m, cudaStream_t stream);

// dst = the Hermitian matrix whose lower triangle is src's (LAPACK 'L'
// convention: the upper triangle and the imaginary part of the diagonal of
// src are not referenced).
void hermitian_from_lower(const Cx<double>* src, long long lds, Cx<double>* dst, long long ldd, int m,
                          cudaStream_t stream);

// out[c] = ||A(:,c)||_2 for `cols` columns of length `rows`.
void column_norms(const Cx<double>* a, long long lda, int rows, int cols, double* out, cudaStream_t stream);

// r(:,c) = hx(:,c) - values[c] * sx(:,c) (plain arithmetic; search residual).
void search_residual(const Cx<double>* hx, const Cx<double>* sx, long long ld, int rows, int cols,
                     const double* values, Cx<double>* r, cudaStream_t stream);

// Fresh certificate (src/pw_core.cpp:579-593): with compensated (Neumaier)
// sums, metric = Re x^H Sx, value = Re x^H Hx / metric; r = fma(-value, Sx, Hx);
// norms[c] = ||r(:,c)||. values/metric/norms are device arrays of `cols`.
void rayleigh_certificate(const Cx<double>* x, const Cx<double>* hx, const Cx<double>* sx, long long ld, int rows,
                          int cols, double* values, double* metric, Cx<double>* r, double* norms, cudaStream_t stream);

// Re x^H Sx per column, compensated (for S-normalisation).
void metric_norms(const Cx<double>* x, const Cx<double>* sx, long long ld, int rows, int cols, double* out,
                  cudaStream_t stream);

// out(i, j) = x_i^H y_j for columns i < cols_a of a and j < cols_b of b, with
// the compensated complex inner product of the strict refinements
// (src/strict_residual_polish.hpp:33-44).
void compensated_inner_matrix(const Cx<double>* a, const Cx<double>* b, long long ld, int rows, int cols_a,
                              int cols_b, Cx<double>* out, long long ldo, cudaStream_t stream);

// dst (cols x rows, ldd) = src^H for src (rows x cols, lds).
void adjoint_block(const Cx<double>* src, long long lds, int rows, int cols, Cx<double>* dst, long long ldd,
                   cudaStream_t stream);

// out(:, c) = fma(alpha[c], d(:, c), x(:, c)) per real component (alpha on the device).
void fma_columns(const double* alpha, const Cx<double>* d, const Cx<double>* x, long long ld, int rows, int cols,
                 Cx<double>* out, cudaStream_t stream);

// x(:,c) *= scale[c]  (scale is a device array).
void scale_columns(Cx<double>* x, long long ld, int rows, int cols, const double* scale, bool reciprocal_sqrt,
                   cudaStream_t stream);

// Kinetic preconditioning of residual columns (src/pw_core.cpp:1386-1400):
// out(i,c) = -r(i,c) * P(T_i, sum_j |x(j,c)|^2 T_j) with P the bounded rational
// kinetic_preconditioner (src/pw_core.cpp:33-47). out may alias r.
void kinetic_precondition(const Cx<double>* r, const Cx<double>* x, long long ld, int rows, int cols,
                          const double* kinetic, Cx<double>* out, long long ldo, cudaStream_t stream);

// Reproducible full-support seed block (src/pw_core.cpp:1027-1043, 1101-1110):
// column j = 0.05 * broad/||broad|| + e_{order[j]}, where broad draws (re, im)
// pairs from the splitmix64 stream seeded 0x6a09e667f3bcc909, starting at draw
// first_draw + 2*rows*j. The draws are counter-based, so columns are independent.
void broad_seed_block(int rows, int cols, unsigned long long first_draw, const int* order, Cx<double>* out,
                      long long ld, cudaStream_t stream);

// dst(rows x cols, ldd) = src(rows x cols, lds).
// dst += src (rows x cols blocks).
void add_block(const Cx<double>* src, long long lds, Cx<double>* dst, long long ldd, int rows, int cols,
               cudaStream_t stream);
void copy_block(const Cx<double>* src, long long lds, Cx<double>* dst, long long ldd, int rows, int cols,
                cudaStream_t stream);

// dst(:, j) = src(:, index[j]) for j < count (index on the device).
void gather_columns(const Cx<double>* src, long long lds, int rows, const int* index, int count, Cx<double>* dst,
                    long long ldd, cudaStream_t stream);

// Zero a (rows x cols) block.
void zero_block(Cx<double>* a, long long lda, int rows, int cols, cudaStream_t stream);

// x(:,c) *= 1/max(norms[c], tiny) where norms[c] > 0 (unit Euclidean columns).
void unit_columns(Cx<double>* x, long long ld, int rows, int cols, const double* norms, cudaStream_t stream);

}  // namespace sdft_b200
