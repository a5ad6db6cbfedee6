/* sdft_b200: B200-native generalized Davidson hot path of Sparse-DFT behind a C ABI.
 *
 * Plain pointers and sizes only. Complex arrays are interleaved (re, im)
 * doubles; blocks are column-major with leading dimension = rows unless a
 * leading dimension is passed. Every call returns an sdft_b200_status; the
 * text of the last failure on the calling thread is read with
 * sdft_b200_last_error. No exception crosses this boundary.
 *
 * Each entry point names the reference interface it replaces (paths relative
 * to the Sparse-DFT source tree).
 */
#ifndef SDFT_B200_H
#define SDFT_B200_H
#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define SDFT_B200_API __attribute__((visibility("default")))
#else
#define SDFT_B200_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  SDFT_B200_OK = 0,
  SDFT_B200_INVALID_ARGUMENT = 1, /* std::invalid_argument in the reference */
  SDFT_B200_OVERFLOW = 2,         /* std::overflow_error */
  SDFT_B200_RUNTIME_ERROR = 3,    /* std::runtime_error (numerical failure) */
  SDFT_B200_CUDA_ERROR = 4,       /* runtime_error("CUDA: ...") / cuBLAS / cuSOLVER */
  SDFT_B200_OUT_OF_MEMORY = 5,    /* std::bad_alloc */
  SDFT_B200_NONFINITE = 6,        /* runtime_error on a nonfinite operator result */
  SDFT_B200_NOT_READY = 7,        /* a served solve has not finished within the wait */
  SDFT_B200_UNSUPPORTED = 8       /* the reference routes this case to a solver not provided here
                                     (indefinite PAW overlap: the caller keeps the reference's route) */
} sdft_b200_status;

enum { SDFT_B200_PRECISION_FP64 = 0, SDFT_B200_PRECISION_MIXED = 1 };
enum { SDFT_B200_MEMORY_HOST = 0, SDFT_B200_MEMORY_DEVICE = 1 };
enum { SDFT_B200_HAMILTONIAN = 0, SDFT_B200_OVERLAP = 1 };

typedef struct sdft_b200_context sdft_b200_context;
typedef struct sdft_b200_operator sdft_b200_operator;

/* Copies the calling thread's last error message; returns its full length. */
SDFT_B200_API size_t sdft_b200_last_error(char* buffer, size_t length);
/* Library version string (static storage). */
SDFT_B200_API const char* sdft_b200_version(void);
/* Number of this library's own CUDA kernels launched by the process so far
 * (cuBLAS/cuSOLVER launches are not counted). No reference counterpart: it
 * backs the benchmark's launch accounting. */
SDFT_B200_API unsigned long long sdft_b200_kernel_launches(void);

/* The tensor-core GEMM tile autotuner's table so far (process-wide): per
 * shape class five values -- rows rounded up to 128, real columns (twice the
 * complex columns) rounded up to 32, K blocks of 64 rounded up to a geometric
 * grid of ratio 2^(1/8), the chosen column tile
 * width and split-K count -- into rows[0 .. 5*capacity). *count receives the
 * number of classes. The first product of a class times each candidate
 * (three tile widths x split counts around the cost model's) on its stream
 * and keeps the fastest; SDFT_B200_GEMM_AUTOTUNE=0 uses the cost model only.
 * No reference counterpart (the reference calls a library ZGEMM). */
SDFT_B200_API sdft_b200_status sdft_b200_gemm_tuned_classes(size_t capacity, int32_t* rows, size_t* count);

/* One CUDA stream + library handles on `device`. `stream` may be NULL (a
 * private non-blocking stream is created) or a cudaStream_t to share.
 * Replaces: make_cuda_accelerator() / class Accelerator, src/compute_backend.hpp:64-91. */
SDFT_B200_API sdft_b200_status sdft_b200_context_create(int device, void* stream, sdft_b200_context** out);
/* Destroying a context releases its buffers and hands the library's unused
 * pooled device memory back to the device. */
SDFT_B200_API sdft_b200_status sdft_b200_context_destroy(sdft_b200_context* context);
/* Device memory of operators, plans and working buffers is stream-ordered
 * memory from one library pool per device; freed blocks stay in the pool for
 * the next allocation (creating and destroying operators then never
 * synchronises the device). This call waits for the context's stream, frees
 * its working buffers (they grow again on demand) and hands every unused
 * block of the pool back to the device, for callers that want the memory for
 * another allocator. Live operators and other contexts keep theirs.
 * No reference counterpart (the reference's accelerator frees on destruction). */
SDFT_B200_API sdft_b200_status sdft_b200_context_release_memory(sdft_b200_context* context);
SDFT_B200_API sdft_b200_status sdft_b200_context_synchronize(sdft_b200_context* context);

/* Plane-wave sphere 1/2|G+k|^2 <= cutoff_ev, sorted by (kinetic, h, k, l);
 * reciprocal rows are b1, b2, b3. Call with capacity 0 to get *count first.
 * Replaces: enumerate_g_vectors, src/pw_core.hpp:17-19 (src/pw_core.cpp:140-171). */
SDFT_B200_API sdft_b200_status sdft_b200_enumerate_g_vectors(const double reciprocal[9], double cutoff_ev, const double kpoint[3],
                                               double hartree_to_ev, int32_t* hkl, double* cartesian,
                                               double* kinetic_ev, size_t capacity, size_t* count);

/* Device-resident H~ = T + V(r) + sum_a B_a^H D_a B_a and
 * S~ = (1+regularization) I + sum_a B_a^H Q_a B_a.
 * hkl: npw x 3 basis indices; kinetic_ev: 1/2|G+k|^2 in eV; potential: V(G)
 * (Hartree) on potential_count keys; per atom a: projectors[a] rows of
 * amplitudes (row-major np_a x npw), D_a and Q_a (row-major np_a x np_a).
 * Replaces: PlaneWaveOperator::PlaneWaveOperator, src/plane_wave_operator.hpp:27-30. */
SDFT_B200_API sdft_b200_status sdft_b200_operator_create(sdft_b200_context* context, size_t npw, const int32_t* hkl,
                                           const double* kinetic_ev, size_t potential_count,
                                           const int32_t* potential_hkl, const double* potential, size_t atoms,
                                           const uint64_t* projectors, const double* amplitudes, const double* d,
                                           const double* q, double hartree_to_ev, double regularization,
                                           sdft_b200_operator** out);
SDFT_B200_API sdft_b200_status sdft_b200_operator_destroy(sdft_b200_operator* op);
/* SCF refresh of a live operator: replaces V(G) (potential_count keys, as in
 * sdft_b200_operator_create) and the per-atom D_a, Q_a (row-major, the
 * operator's projector counts), recomputing V(r) and the H/S diagonals, while
 * the basis maps, FFT plan, B and B's tensor-core packing stay resident. Same
 * checks and arithmetic as sdft_b200_operator_create: the operator afterwards
 * equals one created from the same basis and amplitudes with the new V(G), D
 * and Q, bit for bit (the grid depends on the basis extent alone, since only
 * keys inside it are retained). INVALID_ARGUMENT, with the operator
 * unchanged, when a check fails, when SDFT_FFT_GRID changed since creation so
 * that the grid would differ, or for an operator read from a snapshot (no G
 * components). Synchronous.
 * Replaces: the per-iteration PlaneWaveOperator rebuild that keeps B resident
 * through an immutable projector identity, src/scf_core.cpp:2312-2313
 * (src/plane_wave_operator.cpp:395-397, src/compute_backend.hpp:32-39). */
SDFT_B200_API sdft_b200_status sdft_b200_operator_update(sdft_b200_operator* op, size_t potential_count,
                                                         const int32_t* potential_hkl, const double* potential,
                                                         const double* d, const double* q);

/* Grid shape, grid points, total projector rows, plane waves, and the number
 * of grid rows i0 that hold sphere points (the rows the fused FFT keeps).
 * Replaces: PlaneWaveOperator::fft_grid_points, src/plane_wave_operator.hpp:38. */
SDFT_B200_API sdft_b200_status sdft_b200_operator_info(const sdft_b200_operator* op, int32_t shape[3], size_t* grid_points,
                                         size_t* projectors, size_t* npw, size_t* active_rows);
/* Signature of S~ from its projector block: *minimum = min(1+reg, lowest
 * eigenvalue of (1+reg) I + R Q R) with R = (B B^H)^(1/2), *indefinite =
 * (minimum < -1e-10); RUNTIME_ERROR "original PAW overlap is numerically
 * singular" when |minimum| <= 1e-10 (the outputs are still written). FP64 on
 * the device, computed once per operator (again after an update). The
 * Davidson entry points make the same checks first: singular is that
 * RUNTIME_ERROR, indefinite is UNSUPPORTED (the reference hands such a pencil
 * to its indefinite-metric solver, src/pw_core.cpp:556-557).
 * Replaces: the signature block of PlaneWaveOperator::overlap() and
 * HermitianOperator::indefinite_metric, src/plane_wave_operator.cpp:702-717,
 * src/pw_core.hpp:167. */
SDFT_B200_API sdft_b200_status sdft_b200_operator_metric_signature(sdft_b200_operator* op, double* minimum,
                                                                   int* indefinite);
/* Local part of H~ (y = T o x + (1/N) FFT_fwd(V(r) . FFT_bwd(scatter x))) on
 * DEVICE pointers x, y (npw x columns, ld npw), with no allocation of any
 * kind: the FFT slab and twiddle tables live in a fixed 32 MiB static device
 * array per device, looked up once per device by the first call (which must
 * therefore come before any stream capture on that device). A call whose
 * slab (active rows x n1 x n2 x columns complex values of the precision)
 * exceeds the array is rejected with INVALID_ARGUMENT naming the column
 * limit. Nothing in the array has to start at zero. All calls on one device
 * share the array: calls whose work overlaps in time on different streams,
 * threads or contexts race; calls on one stream are ordered. Same results as
 * sdft_b200_apply_local. For callers that must not allocate (memory reserved
 * up front, or no room for the device-wide synchronisation of cudaFree).
 * x and y must be memory of the operator's device (INVALID_ARGUMENT before
 * any launch otherwise). The array's address belongs to the device's primary
 * context, which the library assumes for the life of the process.
 * No reference counterpart. */
SDFT_B200_API sdft_b200_status sdft_b200_apply_local_noalloc(sdft_b200_operator* op, const double* x,
                                                             size_t columns, double* y, int precision);
/* Sphere-to-grid index map (npw values), T (Hartree), H and S diagonals
 * (npw each), V(r) (grid_points values); any pointer may be NULL.
 * Replaces: the Impl members indices/kinetic/h_diagonal/s_diagonal/local_real,
 * src/plane_wave_operator.cpp:33-34. */
SDFT_B200_API sdft_b200_status sdft_b200_operator_arrays(const sdft_b200_operator* op, uint64_t* indices, double* kinetic,
                                           double* h_diagonal, double* s_diagonal, double* local_potential);

/* y = H~ x or S~ x for `columns` columns (npw x columns). memory selects host
 * or device pointers; host calls are synchronous.
 * Replaces: HermitianOperator::apply_block_into, src/pw_core.hpp:116-117
 * (Impl::apply_block_into, src/plane_wave_operator.cpp:218-306). */
SDFT_B200_API sdft_b200_status sdft_b200_apply(sdft_b200_operator* op, int which, const double* x, size_t columns, double* y,
                                 int precision, int memory);
/* Local part only, y = T x + (1/N) FFT_fwd(V(r) FFT_bwd(x))[idx], on the
 * operator's resident grid maps and V(r). MIXED runs the FFTs and V(r) in FP32.
 * Replaces: Accelerator::local_hamiltonian / accelerated_local_hamiltonian,
 * src/compute_backend.hpp:42-45,81-83 (CPU loop src/plane_wave_operator.cpp:237-257). */
SDFT_B200_API sdft_b200_status sdft_b200_apply_local(sdft_b200_operator* op, const double* x, size_t columns, double* y,
                                                     int precision, int memory);
/* Joint (H~x, S~x) sharing one B x.
 * Replaces: HermitianOperator::apply_pair_into, src/pw_core.hpp:122-124 (src/plane_wave_operator.cpp:307-374). */
SDFT_B200_API sdft_b200_status sdft_b200_apply_pair(sdft_b200_operator* op, const double* x, size_t columns, double* hy,
                                      double* sy, int precision, int memory);
/* P = B x (projectors x columns).
 * Replaces: HermitianOperator::project_into, src/pw_core.hpp:130-131 (src/plane_wave_operator.cpp:375-380). */
SDFT_B200_API sdft_b200_status sdft_b200_project(sdft_b200_operator* op, const double* x, size_t columns, double* p,
                                   int precision, int memory);

/* Accelerator-style local part on caller arrays (no resident operator):
 * output = kinetic o input + (1/N) FFT_fwd(potential . FFT_bwd(scatter(input)))[indices]
 * for `columns` columns of npw values; potential holds the real V(r) on the
 * shape[0] x shape[1] x shape[2] grid (row-major). A nonzero operator_identity
 * promises immutable shape/indices/potential for that identity, so the device
 * copies are reused; zero re-uploads them. kinetic and input are per call.
 * Replaces: Accelerator::local_hamiltonian, src/compute_backend.hpp:81-83
 * (accelerated_local_hamiltonian, src/compute_backend.hpp:42-45). */
SDFT_B200_API sdft_b200_status sdft_b200_local_hamiltonian(sdft_b200_context* context, const int32_t shape[3],
                                                           const uint64_t* indices, size_t npw, const double* kinetic,
                                                           const double* potential, const double* input,
                                                           size_t columns, double* output, int precision,
                                                           uint64_t operator_identity);
/* PAW chain on caller arrays: h = B^H (D (B x)), s = B^H (Q (B x)) with B the
 * projectors x npw column-major matrix and D, Q dense projectors x projectors.
 * A nonzero projector_identity keeps B resident (and its tensor-core packing);
 * a nonzero identity keeps D and Q resident. Host pointers, synchronous.
 * Replaces: Accelerator::paw_pair, src/compute_backend.hpp:87-88
 * (accelerated_paw_pair, src/compute_backend.hpp:48-50). */
SDFT_B200_API sdft_b200_status sdft_b200_paw_pair(sdft_b200_context* context, uint64_t identity, size_t npw,
                                                  size_t projectors, size_t columns, const double* b, const double* d,
                                                  const double* q, const double* input, double* h, double* s,
                                                  int precision, uint64_t projector_identity);

/* Spin-unpolarised PBE per point in FP64: for density n > 0 and gradient
 * magnitude |grad n| >= 0, out[7*i ..] = energy density, energy per particle,
 * exchange energy density, correlation energy density, exchange potential,
 * correlation potential, 2 dE/d|grad n|^2 coefficient (the PbeXcPoint fields).
 * Invalid points give INVALID_ARGUMENT, nonfinite results NONFINITE.
 * Replaces: Accelerator::pbe_points / accelerated_pbe_points,
 * src/compute_backend.hpp:46-47,84-86 (pbe_unpolarized, src/pbe_xc.cpp:116-140). */
SDFT_B200_API sdft_b200_status sdft_b200_pbe_points(sdft_b200_context* context, const double* density,
                                                    const double* gradient, size_t count, double* out, int memory);

/* Band density on a Fourier support, FP64:
 * out[j] = (1/N) FFT_fwd( sum_b occupations[b]/volume |FFT_bwd(scatter psi_b)|^2 )[support_j]
 * psi: `bands` x npw complex (interleaved re, im), band-major (band b at
 * psi + 2*b*npw); hkl: npw keys (h,k,l) of the plane waves; support: `count`
 * keys; out: `count` complex values in support order. The density grid is the
 * reference's alias-free rule max(3, 2m+1) per axis, rounded up to a
 * 2/3/5/7-smooth length (its SDFT_FAST_DENSITY_GRID=1 option). hkl, support
 * and occupations are host arrays; psi and out follow `memory`.
 * Occupations outside [0,2] or nonfinite, nonfinite coefficients of occupied
 * bands, empty inputs and duplicate plane-wave keys give INVALID_ARGUMENT.
 * Replaces: plane_wave_density_fft, src/density_functionals.hpp:15-19
 * (src/density_functionals.cpp:407-460). */
SDFT_B200_API sdft_b200_status sdft_b200_band_density(sdft_b200_context* context, const int32_t* hkl, size_t npw,
                                                      const double* psi, const double* occupations, size_t bands,
                                                      double volume, const int32_t* support, size_t count,
                                                      double* out, int memory);

/* One-centre occupations of `atoms` atoms with `rows` projectors each:
 * out[a][i][j] = sum_n occupations[n] P[a*rows+i, n] conj(P[a*rows+j, n])
 * (row-major rows x rows per atom). amplitudes: (atoms*rows) x bands complex,
 * column-major with column stride `stride` >= atoms*rows (the all-atom FP64
 * projection B psi); occupations: host, in [0, 2]. amplitudes and out follow
 * `memory`. Replaces: onsite_density_from_amplitudes, src/onsite_density.hpp:10-36
 * (called per atom on a row view of one projection). */
SDFT_B200_API sdft_b200_status sdft_b200_onsite_density(sdft_b200_context* context, size_t rows, size_t atoms,
                                                        size_t bands, const double* amplitudes, size_t stride,
                                                        const double* occupations, double* out, int memory);

/* Compensation charge of atoms sharing one PAW augmentation on a reciprocal
 * support. create: lattice (3 lattice vectors as rows, bohr), fractional atom
 * positions (atoms x 3), keys (count x 3), the radial mesh (Angstrom) and
 * g_L(r) r^2 shapes ((max_l+1) x radial), and the (L,M) transform of the
 * one-centre occupation ((max_l+1)^2 x dimension^2 complex, entry
 * [LM][i*dimension+j] = the LM moment of the unit occupation at (i,j), i.e.
 * the reference's density_transform_). Form factors are integrated on the
 * device at creation. All host arrays; copied. density: onsite is atoms x
 * dimension^2 complex row-major Hermitian occupations, out is count complex
 * values in key order; both follow `memory`.
 * Replaces: PawCompensationOperator(augmentation, lattice, position, keys,
 * Codata, shared) and PawCompensationOperator::density_sum,
 * src/paw_compensation.hpp:14-27 (src/paw_compensation.cpp:185-342,465-524). */
typedef struct sdft_b200_compensation sdft_b200_compensation;
SDFT_B200_API sdft_b200_status sdft_b200_compensation_create(
    sdft_b200_context* context, const double lattice[9], size_t atoms, const double* fractional,
    const int32_t* keys, size_t count, int max_l, size_t radial, const double* radial_grid,
    const double* compensation_r2, size_t dimension, const double* transform, sdft_b200_compensation** out);
SDFT_B200_API sdft_b200_status sdft_b200_compensation_destroy(sdft_b200_compensation* charge);
SDFT_B200_API sdft_b200_status sdft_b200_compensation_density(sdft_b200_compensation* charge, const double* onsite,
                                                              double* out, int memory);
/* The adjoint: potential (V(G) on the charge's support keys, in their order;
 * a mode absent from the potential is 0), out (atoms x dimension^2 row-major)
 * = sum_LM [sum_G V(-G) e^{-iG.tau_a} F_LM(G)] T_LM, the (L,M) transform T.
 * Replaces: PawCompensationOperator::project_potential_batch, src/paw_compensation.cpp:552-629. */
SDFT_B200_API sdft_b200_status sdft_b200_compensation_project(sdft_b200_compensation* charge, const double* potential,
                                                              double* out, int memory);

/* Hartree + PBE exchange-correlation functional of a Fourier density
 * n(r) = sum_G n_G exp(+iG.r) on one device, with the reference's default
 * packing (paired real transforms, fused PBE tiles, fixed-tile reductions).
 * lattice: rows a1, a2, a3 (bohr). density: `count` keys hkl (x3) and values
 * (interleaved complex), unique, any order; core: the optional frozen
 * pseudo-core (core_count 0 for none), added for XC only. quadrature_padding
 * 0 takes SDFT_FFT_OVERSAMPLING or 2; the XC grid is padding * max(3, 2m+1)
 * per axis (any length up to 512; SDFT_FAST_DENSITY_GRID=1 rounds it up to a
 * 2/3/5/7-smooth length). Outputs on the union support of density and core
 * in the reference's map order (lexicographic h, k, l): support_hkl (x3),
 * potential = Hartree (density keys, 0 at G = 0) + v_xc, and xc_potential =
 * v_xc (interleaved complex). Call with capacity 0 to get *support_count
 * (host only: context may be NULL, and the host checks run); capacity below
 * it is INVALID_ARGUMENT. The
 * scalars agree with the reference to rounding (double-double sums where it
 * sums long double). Host pointers, synchronous.
 * Replaces: evaluate_density_functionals, src/density_functionals.hpp:45-47
 * (src/density_functionals.cpp:462-729). */
typedef struct {
  double hartree_energy, xc_energy, vxc_density;
  double hartree_stress[9], xc_stress[9]; /* row-major 3 x 3 */
  double sampled_electrons, minimum_density;
  uint64_t clipped_density_points, grid_points;
  int32_t grid[3];
} sdft_b200_functionals;
SDFT_B200_API sdft_b200_status sdft_b200_density_functionals(
    sdft_b200_context* context, const double lattice[9], size_t count, const int32_t* hkl, const double* density,
    size_t core_count, const int32_t* core_hkl, const double* core, int quadrature_padding, int32_t* support_hkl,
    double* potential, double* xc_potential, size_t capacity, size_t* support_count, sdft_b200_functionals* result);

/* Collinear spin form on one device: up and down channel densities (each
 * `count` keys and values, unique), the optional frozen core (each channel
 * receives half of it for XC), padding 0 = SDFT_FFT_OVERSAMPLING or 2. Per
 * channel: potential = Hartree of the total density + that channel's v_xc,
 * xc_potential = v_xc (collinear PBE with PW92 spin interpolation), and
 * result[c] with the Hartree and XC energies and stresses split equally,
 * <n_c, v_xc,c>, electrons Omega Re n_c(0), the channel's minimum and its
 * count of negative samples (clipped_density_points). Outputs on the union
 * support of both channels and the core in map order; capacity 0 queries
 * *support_count on the host (context may be NULL).
 * Replaces: evaluate_collinear_density_functionals, src/density_functionals.hpp:52-56
 * (src/density_functionals.cpp:732-806; pbe_collinear, src/spin_pbe_xc.cpp:54-107). */
SDFT_B200_API sdft_b200_status sdft_b200_collinear_functionals(
    sdft_b200_context* context, const double lattice[9], size_t count_up, const int32_t* hkl_up, const double* up,
    size_t count_down, const int32_t* hkl_down, const double* down, size_t core_count, const int32_t* core_hkl,
    const double* core, int padding, int32_t* support_hkl, double* potential_up, double* potential_down,
    double* xc_potential_up, double* xc_potential_down, size_t capacity, size_t* support_count,
    sdft_b200_functionals result[2]);

/* Rayleigh-Ritz eigensolve of a projected pencil in FP64: the lowest
 * `requested` (0 = all n) solutions of H y = e S y, H and S n x n Hermitian
 * (lower triangles referenced, column-major), S positive definite. values:
 * count = requested ? requested : n ascending eigenvalues; vectors: n x count
 * column-major, S-orthonormal. For S within 1e-5 of the identity the device
 * eigensolver runs (Householder tridiagonalisation in one cooperative
 * kernel, multisection, inverse iteration, compact-WY back-transform) after a
 * first- or second-order Loewdin reduction; otherwise, or for n above the
 * device solver's limit, cuSOLVER zhegvdx/zhegvd. memory applies to h, s, values and vectors.
 * Replaces: rayleigh_ritz(h, s, requested), src/pw_core.cpp:56-136. */
SDFT_B200_API sdft_b200_status sdft_b200_rayleigh_ritz(sdft_b200_context* context, size_t n, size_t requested,
                                                       const double* h, const double* s, double* values,
                                                       double* vectors, int memory);

enum { SDFT_B200_OP_NORMAL = 0, SDFT_B200_OP_ADJOINT = 1 };

/* C(m x n, ldc) = op(A) op(B) (+ C when add), column-major complex with
 * explicit leading dimensions. FP64: FP64 arithmetic (cuBLAS ZGEMM). MIXED:
 * BF16 split products on the tcgen05 tensor cores with FP32 accumulation (an
 * ADJOINT right operand is formed as B^H on the device first). memory applies
 * to a, b and c.
 * Replaces: complex_gemm(MatrixOp, MatrixOp, m, n, k, a, lda, b, ldb, c, ldc, exact, add),
 * src/compute_backend.hpp:23-26 (exact=true -> FP64, exact=false -> MIXED). */
SDFT_B200_API sdft_b200_status sdft_b200_complex_gemm(sdft_b200_context* context, int aop, int bop, size_t m,
                                                      size_t n, size_t k, const double* a, size_t lda,
                                                      const double* b, size_t ldb, double* c, size_t ldc,
                                                      int precision, int add, int memory);

/* C(m x n, ldc) = op(A) B (+ C when add) for a left operand A that the caller
 * promises immutable for `identity` (nonzero, e.g. from the reference's
 * new_immutable_matrix_identity()): A (op(A) m x k; stored rows x cols with
 * leading dimension lda) is copied to the device on the first call for that
 * identity and operation and reused afterwards (MIXED also keeps its
 * tensor-core packing); B (k x n, ldb) and C are dynamic. Four operands stay
 * cached per context, least recently used replaced. A changed A must come
 * with a new identity: the cache never re-reads it.
 * Replaces: Accelerator::gemm_immutable_left / complex_gemm_immutable_left,
 * src/compute_backend.hpp:32-41,68-71 (src/compute_backend.cpp:87-100). */
SDFT_B200_API sdft_b200_status sdft_b200_complex_gemm_immutable_left(sdft_b200_context* context, uint64_t identity,
                                                                     int aop, size_t m, size_t n, size_t k,
                                                                     const double* a, size_t lda, const double* b,
                                                                     size_t ldb, double* c, size_t ldc, int precision,
                                                                     int add, int memory);

/* C_i(m x n, ldc) = A_i B for i = 0, 1, 2 (A_i m x k with leading dimension
 * lda, B k x n with ldb shared: staged once). Outputs must not overlap B, the
 * A_i or each other (INVALID_ARGUMENT, as the reference checks). FP64, or the
 * tensor-core split products for MIXED.
 * Replaces: Accelerator::gemm_triple_right / complex_gemm_triple_right,
 * src/compute_backend.hpp:72-77, src/compute_backend.cpp:255-332. */
SDFT_B200_API sdft_b200_status sdft_b200_complex_gemm_triple_right(sdft_b200_context* context, size_t m, size_t n,
                                                                   size_t k, const double* const a[3], size_t lda,
                                                                   const double* b, size_t ldb, double* const c[3],
                                                                   size_t ldc, int precision, int memory);

/* Davidson controls. precision selects the search arithmetic (MIXED: FP32
 * FFT/V_loc and FP32-accumulated projector and subspace products; FP64: the
 * plain form throughout); Rayleigh-Ritz, the FP64 refresh and the final
 * certificate are FP64 on the device in both. subspace_factor in [4,16]
 * (capacity = min(npw, max(factor*roots, 64)); 0 selects 8). handoff: search
 * residual below which the basis is re-applied in FP64 (0 selects 1e-8).
 * correction_steps (MIXED only): how the basis is expanded. The reference
 * expands with the kinetic preconditioner applied once to each residual
 * (src/pw_core.cpp:1384-1401); a positive value runs that many steps of
 * preconditioned CG on each unconverged root's Jacobi-Davidson correction
 * equation instead (mixed-form applies, tensor-core projections), which
 * needs far fewer outer iterations; 0 selects the library's default for
 * MIXED (SDFT_B200_CORRECTION_STEPS, else 6); -1 keeps the reference's
 * single preconditioner step. FP64 solves take 0 (the reference's step). */
typedef struct {
  size_t roots;
  size_t max_iterations;
  double tolerance;
  int precision;
  int subspace_factor;
  double handoff;
  int correction_steps;
} sdft_b200_davidson_options;

typedef struct {
  size_t iterations;
  int converged;
  double max_residual;
  double seconds;
  double rayleigh_ritz_seconds;
  size_t h_columns_search, h_columns_fp64, s_columns_search, s_columns_fp64;
  int rayleigh_ritz_calls, restarts, fp64_refreshes, certifications, handoff_iteration, block_rank_fallbacks;
  size_t correction_columns; /* mixed-form pair applies spent on Jacobi-Davidson corrections, in columns */
  /* strict FP64 refinements (src/strict_residual_polish.hpp): tangent polish
   * steps tried / accepted, root-manifold steps tried / accepted */
  int polish_steps, polish_accepted, manifold_steps, manifold_accepted;
} sdft_b200_davidson_stats;

/* Lowest `roots` eigenpairs of H~ x = e S~ x. initial: band-major roots x npw
 * warm vectors or NULL; eigenvectors: band-major roots x npw output (may be
 * NULL); residuals: fresh FP64 ||H~x - e S~x|| per root. memory applies to
 * initial/eigenvectors (eigenvalues, residuals and stats are host memory).
 * A solve that exhausts max_iterations returns OK with stats->converged = 0
 * and its fresh residuals, as the reference does.
 * Replaces: solve_generalized_hermitian_davidson(const HermitianOperator&, const HermitianOperator&,
 * size_t, size_t, double, const std::vector<std::complex<double>>&), src/pw_core.hpp:184-188. */
SDFT_B200_API sdft_b200_status sdft_b200_davidson(sdft_b200_operator* op, const sdft_b200_davidson_options* options,
                                                  const double* initial, double* eigenvalues, double* eigenvectors,
                                                  double* residuals, sdft_b200_davidson_stats* stats, int memory);

/* Residual-minimisation trial for SCF warm solves: at most
 * min(16, max_iterations/2) steps of global rotation, preconditioned
 * directions and a per-band 2 x 2 residual minimisation from the warm block
 * `initial` (band-major roots x npw, required); tolerance must be coarse
 * (> 1e-9). A block whose fresh FP64 residuals meet the tolerance and is
 * S-orthonormal within 1e-10 returns with *trial_manifold = 1 and
 * stats->converged = 0 (a residual-checked trial, explicitly not a converged
 * lowest spectrum); otherwise the Davidson solve continues from the trial's
 * block with the remaining iterations (*trial_manifold = 0) and its result is
 * returned, iterations counted in total. Directions are applied in FP64 for
 * tolerances below 1e-6, in the mixed form otherwise.
 * Replaces: solve_generalized_hermitian_rmm_trial, src/pw_core.hpp:170-178
 * (src/rmm_trial.cpp:128-206; selected by SDFT_SCF_RMM_TRIAL=1 for SCF warm
 * requests, src/pw_core.cpp:558-563). */
SDFT_B200_API sdft_b200_status sdft_b200_rmm_trial(sdft_b200_operator* op, const sdft_b200_davidson_options* options,
                                                   const double* initial, double* eigenvalues, double* eigenvectors,
                                                   double* residuals, sdft_b200_davidson_stats* stats,
                                                   int* trial_manifold, int memory);

/* Band-group solve: groups of SDFT_BAND_GROUP_SIZE (default 8) bands solved
 * in turn by local Davidson solves (capacity 5 x group size) deflated
 * against the S-orthonormalised completed bands, then a roots x roots
 * Rayleigh-Ritz rotation of the whole block and fresh FP64 residuals; two
 * sweeps, or with SDFT_BAND_GROUP_SWEEP=1 3-iteration local searches within
 * half the budget and a global Davidson solve for the rest. initial: band-major
 * roots x npw warm vectors or NULL. Returns OK with stats->converged = 0 when
 * the sweeps end uncertified, as the reference does.
 * Replaces: solve_generalized_hermitian_band_groups, src/pw_core.hpp:179-182
 * (src/band_group_solver.cpp:55-212; SDFT_BAND_GROUP_SOLVER=1, src/pw_core.cpp:564-567). */
SDFT_B200_API sdft_b200_status sdft_b200_band_groups(sdft_b200_operator* op, const sdft_b200_davidson_options* options,
                                                     const double* initial, double* eigenvalues, double* eigenvectors,
                                                     double* residuals, sdft_b200_davidson_stats* stats, int memory);

/* ---- Solver snapshots ------------------------------------------------------
 * The reference's SDFTPWO3 files (PlaneWaveOperator::save_solver_snapshot,
 * src/plane_wave_operator.cpp:542-569; replayed by sdft_solver_replay):
 * the operator's internal arrays and the solve settings. */
typedef struct {
  size_t npw, grid_points, projectors, atoms, roots, iterations, initial_values;
  int32_t shape[3];
  double regularization, tolerance;
} sdft_b200_snapshot_info;

/* Header fields after the reference's checks (host only, no device).
 * Replaces: the header checks of PlaneWaveOperator::load_solver_snapshot,
 * src/plane_wave_operator.cpp:571-604. */
SDFT_B200_API sdft_b200_status sdft_b200_snapshot_read_info(const char* path, sdft_b200_snapshot_info* info);
/* Device operator from a snapshot; initial (band-major roots x npw, host,
 * may be NULL) receives the snapshot's warm vectors when it has them.
 * Replaces: PlaneWaveOperator::load_solver_snapshot, src/plane_wave_operator.cpp:571-653. */
SDFT_B200_API sdft_b200_status sdft_b200_operator_from_snapshot(sdft_b200_context* context, const char* path,
                                                                sdft_b200_operator** out, double* initial);

/* ---- Solve server: continuous batching of independent solves ------------
 * One request = one operator (one cell, one k-point) and its Davidson solve,
 * copied in at submit. Requests wait in a FIFO queue and start when a worker
 * slot is free and their estimated device footprint fits under memory_cap
 * beside the solves already running; each worker owns a stream, cuBLAS and
 * cuSOLVER handles and scratch, so admitted solves overlap on the device and
 * each result is the one the request gives alone. The operator and Davidson
 * state of a running solve stay resident until it finishes.
 * Replaces: the concurrent k-team solves over distinct operators
 * (src/scf_core.cpp:2974-3061), one PlaneWaveOperator + solve per team. */
typedef struct sdft_b200_server sdft_b200_server;

typedef struct {
  int slot;                           /* worker that ran the solve */
  size_t footprint;                   /* budgeted device bytes */
  double submitted, started, finished; /* seconds since the server started */
} sdft_b200_solve_timing;

SDFT_B200_API sdft_b200_status sdft_b200_server_create(int device, uint64_t memory_cap, int slots,
                                                       sdft_b200_server** out);
/* Waits for the running solves; requests still queued are answered with an error. */
SDFT_B200_API sdft_b200_status sdft_b200_server_destroy(sdft_b200_server* server);
/* Arguments as sdft_b200_operator_create and sdft_b200_davidson (host
 * arrays). INVALID_ARGUMENT when the footprint exceeds the cap. */
SDFT_B200_API sdft_b200_status sdft_b200_server_submit(sdft_b200_server* server, size_t npw, const int32_t* hkl,
                                                       const double* kinetic_ev, size_t potential_count,
                                                       const int32_t* potential_hkl, const double* potential,
                                                       size_t atoms, const uint64_t* projectors,
                                                       const double* amplitudes, const double* d, const double* q,
                                                       double hartree_to_ev, double regularization,
                                                       const sdft_b200_davidson_options* options, int want_vectors,
                                                       uint64_t* ticket);
/* Waits up to timeout seconds (negative: no limit). NOT_READY when the solve
 * is still queued or running; otherwise the solve's own status (its message
 * through sdft_b200_last_error), with the outputs of sdft_b200_davidson
 * (host memory; eigenvectors only when requested at submit, may be NULL). */
SDFT_B200_API sdft_b200_status sdft_b200_server_wait(sdft_b200_server* server, uint64_t ticket, double timeout,
                                                     double* eigenvalues, double* eigenvectors, double* residuals,
                                                     sdft_b200_davidson_stats* stats,
                                                     sdft_b200_solve_timing* timing);
SDFT_B200_API sdft_b200_status sdft_b200_server_memory(const sdft_b200_server* server, uint64_t* cap,
                                                       uint64_t* in_use, uint64_t* peak);
/* The device bytes a solve is budgeted at by the server's admission. */
SDFT_B200_API sdft_b200_status sdft_b200_solve_footprint(size_t npw, const int32_t* hkl, size_t projectors_total,
                                                         size_t roots, int subspace_factor, uint64_t* bytes);

#ifdef __cplusplus
}
#endif
#endif
