/* FFTW3-API declarations for the oracle build (test infrastructure only).
 *
 * The reference sources (src/plane_wave_operator.cpp, src/density_functionals.cpp,
 * src/fft_planning.hpp) call FFTW3, which is not installed in this image. This
 * header declares exactly the subset they call, with the FFTW3 public names and
 * argument meanings, so the reference's own translation units compile unmodified.
 * The implementation (fftw_shim.cpp) is this project's mixed-radix FFT, written
 * from the DFT definition: unnormalised, X_k = sum_j x_j exp(sign*2*pi*i*j*k/n),
 * sign = -1 for FFTW_FORWARD and +1 for FFTW_BACKWARD, row-major multi-dimensional
 * layout. Nothing here is FFTW code.
 */
#ifndef SDFT_ORACLE_FFTW3_SHIM_H
#define SDFT_ORACLE_FFTW3_SHIM_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef double fftw_complex[2];
typedef struct sdft_oracle_fft_plan* fftw_plan;
#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_PATIENT (1U << 5)
#define FFTW_EXHAUSTIVE (1U << 3)
fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex* in, fftw_complex* out,
                           int sign, unsigned flags);
fftw_plan fftw_plan_many_dft(int rank, const int* n, int howmany, fftw_complex* in,
                             const int* inembed, int istride, int idist, fftw_complex* out,
                             const int* onembed, int ostride, int odist, int sign,
                             unsigned flags);
void fftw_execute(const fftw_plan plan);
void fftw_execute_dft(const fftw_plan plan, fftw_complex* in, fftw_complex* out);
void fftw_destroy_plan(fftw_plan plan);
fftw_complex* fftw_alloc_complex(size_t n);
void fftw_free(void* p);
int fftw_init_threads(void);
void fftw_plan_with_nthreads(int nthreads);
#ifdef __cplusplus
}
#endif
#endif
