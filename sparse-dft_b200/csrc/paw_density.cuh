// One-centre occupations and the PAW compensation charge on a Fourier
// support, on the device: the reference's onsite_density_from_amplitudes
// (src/onsite_density.hpp:10-36) and PawCompensationOperator with shared
// geometry (constructor src/paw_compensation.cpp:185-342, density_sum :465-524).
#pragma once
#include <cstdint>
#include <vector>

#include "common.cuh"

namespace sdft_b200 {

struct Context;

// rho_a(i,j) = sum_n f_n P(a*rows+i, n) conj(P(a*rows+j, n)) for each atom a,
// row-major rows x rows per atom. P: device, column stride `stride`
// (>= atoms*rows); occupations: host; out: device, atoms*rows*rows values.
void onsite_density(Context& ctx, std::size_t rows, std::size_t atoms, std::size_t bands, const Cx<double>* amplitudes,
                    std::size_t stride, const double* occupations, Cx<double>* out);

struct CompensationInput {
  const double* lattice = nullptr;     // 3 lattice vectors (rows), bohr
  std::size_t atoms = 0;
  const double* fractional = nullptr;  // atoms x 3
  const std::int32_t* keys = nullptr;  // count x 3 reciprocal keys (h, k, l)
  std::size_t count = 0;
  int max_l = 0;
  std::size_t radial = 0;
  const double* radial_grid = nullptr;      // radial points, Angstrom
  const double* compensation_r2 = nullptr;  // (max_l+1) x radial: g_L(r) r^2
  std::size_t dimension = 0;                // expanded one-centre dimension
  const double* transform = nullptr;  // (max_l+1)^2 x dimension^2 complex: (L,M) moments of unit occupations
};

// Device-resident compensation geometry shared by all atoms: reciprocal
// vectors, integer keys, compact form factors F_LM(G) (signed real; i times
// it for odd L), fractional positions and the (L,M) transform. density() evaluates
// rho^(G) = sum_a exp(-i G.tau_a)/Omega sum_LM F_LM(G) M_a,LM with
// M_a = transform . rho_a, in atom order per G.
class CompensationCharge {
 public:
  CompensationCharge(Context& ctx, const CompensationInput& input);
  ~CompensationCharge();
  CompensationCharge(const CompensationCharge&) = delete;
  CompensationCharge& operator=(const CompensationCharge&) = delete;

  // onsite: device, atoms x dimension^2 row-major Hermitian; out: device, count values.
  void density(const Cx<double>* onsite, Cx<double>* out);
  // The adjoint (the reference's project_potential_batch,
  // src/paw_compensation.cpp:552-629): potential: device, count values on
  // the support (V(G) in key order; a mode absent from the potential is 0);
  // out: device, atoms x dimension^2 row-major,
  // out_a = sum_LM [sum_G V(-G) e^{-iG.tau_a} F_LM(G)] transform_LM.
  void project(const Cx<double>* potential, Cx<double>* out);
  std::size_t count() const { return count_; }
  std::size_t atoms() const { return atoms_; }
  std::size_t dimension() const { return dim_; }
  int multipoles() const { return lms_; }
  Context& context() const { return ctx_; }
  // Compact form factors, (L,M)-major: form[lm * count + g] (device).
  const double* form() const { return form_; }

 private:
  Context& ctx_;
  std::size_t count_ = 0, atoms_ = 0, dim_ = 0;
  int lms_ = 0, max_l_ = 0;
  double volume_ = 0;
  double* q_ = nullptr;          // count x 3 cartesian G, 1/bohr
  int* keys_ = nullptr;          // count x 3 integer keys
  double* fractional_ = nullptr; // atoms x 3 fractional positions
  double* form_ = nullptr;       // lms x count
  Cx<double>* transform_ = nullptr;
  Cx<double>* moments_ = nullptr;  // atoms x lms
  unsigned int* flags_ = nullptr;
  int* opposite_ = nullptr;         // index of -G in the support, or -1
  Cx<double>* partials_ = nullptr;  // per-CTA sums of the adjoint
  Cx<double>* responses_ = nullptr; // atoms x lms
};

}  // namespace sdft_b200
