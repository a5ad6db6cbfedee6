// Fused local part of H~: y = T o x + (1/N) FFT_fwd( V(r) . FFT_bwd( scatter(x) ) )[idx]
// for a block of plane-wave columns, plus full-grid 3D FFTs on device grids.
#pragma once
#include <vector>

#include "fft.cuh"

namespace sdft_b200 {

// Device-resident description of a plane-wave sphere inside an n0 x n1 x n2
// grid (row-major index (i0*n1 + i1)*n2 + i2, the reference's layout,
// src/plane_wave_operator.cpp:94-97). Only grid rows i0 that hold sphere
// points ("slots") are ever materialised between the plane and pencil passes.
struct SpherePlan {
  int n[3] = {0, 0, 0};
  std::size_t count = 0;   // n0*n1*n2
  int npw = 0;
  int slots = 0;           // active i0 rows
  int krows = 0;           // active i1 rows (union over slots)
  int n2p = 0;             // padded (odd) shared-memory row stride
  int* slot_row = nullptr;      // [slots]
  int* point_offset = nullptr;  // [slots+1]
  int* point_g = nullptr;       // [npw] plane-wave index, grouped by slot
  int* point_smem = nullptr;    // [npw] i1*n2p + i2
  int* point_compact = nullptr; // [npw] k*n2 + i2, k = position of i1 in krow
  int* krow = nullptr;          // [krows]
  LinePlan line[3];
  std::vector<int> slot_of_row_host;       // [n0] slot of grid row i0, or -1
  std::vector<int> krow_host;              // [krows] the active i1 rows
  std::vector<Cx<float>> twiddles_host[3]; // [n[a]] FP32 twiddles, passed as kernel parameters

  cudaStream_t stream = nullptr;  // the device arrays are stream-ordered pool memory on it

  // Device arrays are allocated and uploaded on `stream` (stream-ordered).
  void build(const int shape[3], const std::vector<std::uint64_t>& indices, cudaStream_t stream);
  void release();
  std::size_t slab_elements(std::size_t columns) const {
    return static_cast<std::size_t>(slots) * n[1] * n[2] * columns;
  }
};

// Local H part for `columns` FP64 input columns (x, ld ldx) into FP64 output
// y (ld ldy). T selects the FFT/V precision (float = mixed search, double =
// FP64 plain form). `slab` must hold plan.slab_elements(columns) Cx<T>.
// potential: V(r) in precision T (plan.count values). kinetic: T(G) Hartree.
template <typename T>
void local_hamiltonian(const SpherePlan& plan, const Cx<double>* x, long long ldx, int columns,
                       const T* potential, const double* kinetic, Cx<double>* y, long long ldy,
                       Cx<T>* slab, cudaStream_t stream);

// local_hamiltonian with caller-provided twiddle tables (twiddle[a] holds
// plan.n[a] values) and slab; launches kernels only, allocates nothing.
template <typename T>
void local_hamiltonian_preset(const SpherePlan& plan, const Cx<double>* x, long long ldx, int columns,
                              const T* potential, const double* kinetic, Cx<double>* y, long long ldy,
                              Cx<T>* slab, const Cx<T>* const twiddle[3], cudaStream_t stream);

// In-place unnormalised 3D FFT of `batch` contiguous row-major grids. Axis
// lengths up to 512; with general = true any length (odd prime factors above
// 7 run the two-pass prime stage), else 2/3/5/7-smooth lengths only.
template <typename T>
void fft3d(Cx<T>* grid, const int n[3], int batch, bool backward, cudaStream_t stream, bool general = false);

}  // namespace sdft_b200
