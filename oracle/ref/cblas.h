/* CBLAS declarations for the oracle build (test infrastructure only).
 *
 * The reference's compute_backend.cpp includes <cblas.h> when SDFT_HAS_CBLAS is
 * set. No CBLAS header is installed in this image, but an LP64 OpenBLAS shared
 * library that exports these symbols ships inside a Python wheel. This header
 * declares the two routines the reference calls, with the standard CBLAS enum
 * values (the numbers are part of the CBLAS calling convention).
 */
#ifndef SDFT_ORACLE_CBLAS_DECLS_H
#define SDFT_ORACLE_CBLAS_DECLS_H
#ifdef __cplusplus
extern "C" {
#endif
enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
void cblas_zgemm(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE transa, enum CBLAS_TRANSPOSE transb,
                 int m, int n, int k, const void* alpha, const void* a, int lda, const void* b,
                 int ldb, const void* beta, void* c, int ldc);
void cblas_dgemm(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE transa, enum CBLAS_TRANSPOSE transb,
                 int m, int n, int k, double alpha, const double* a, int lda, const double* b,
                 int ldb, double beta, double* c, int ldc);
void openblas_set_num_threads(int threads);
#ifdef __cplusplus
}
#endif
#endif
