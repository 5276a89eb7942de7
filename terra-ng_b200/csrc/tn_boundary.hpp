// Launchers of boundary.cu: right-hand-side boundary treatment, the normal-tangential rotation, the
// free-slip/free-slip null-space penalty, and the vector swap. Asynchronous on `st`; 0 or -1 on a launch error.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "tn_grid.hpp"  // ShellBoundaryFlag values kFlag*

namespace tn {

// penalty epsilon of EpsilonDivDivKerngen (epsilon_divdiv_kerngen.hpp:168)
constexpr double kPenaltyEpsilon = 1e-7;
constexpr int    kPenaltyBlocks  = 296;

template <typename T>
struct Ptrs4 {
    T* p[4] = {nullptr, nullptr, nullptr, nullptr};
};

// v[c][i] = m value + (1 - m) v[c][i], m = 1 on nodes whose flags contain `flag` (flag 0: unflagged nodes only)
template <typename T>
int assign_masked(int64_t n, int nr, int ncomp, T* const* v, int flag, T value, cudaStream_t st);
// on nodes carrying `flag`: mode 0 cartesian -> normal-tangential, 1 back, 2 remove the normal component
template <typename T>
int rotate_normal_tangential(int64_t n, int nr, const T* coords, T* const* v, int flag, int mode, cudaStream_t st);
// orthonormal rotation modes n_i = sum_a c[3 i + a] m_a in terms of the raw modes m_a = e_a x X
struct PenaltyCoef {
    double c[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
};
// doubles of per-block partials penalty_gram / penalty_apply need
int penalty_partials_size();
// owned-node Gram matrix of the raw modes, gram[0..5] = <m_a, m_b> for ab = 00 01 02 11 12 22 (FP64, on the
// device; 2 launches)
int penalty_gram(int64_t n, int nr, const uint8_t* owned_lat, const double* coords, const double* radii,
                 double* partials, double* gram, cudaStream_t st);
// dst += eps sum_i <src, n_i>_owned n_i with n_i from coef (3 launches; beta[0..2], the raw-mode coefficients,
// left on the device)
template <typename T>
int penalty_apply(int64_t n, int nr, const uint8_t* owned_lat, const T* coords, const T* radii, const T* const* src,
                  T* const* dst, const PenaltyCoef& coef, double eps, double* partials, double* beta, cudaStream_t st);
// a <-> b elementwise, ncomp components
template <typename T>
int swap_vectors(int64_t n, int ncomp, T* const* a, T* const* b, cudaStream_t st);

}  // namespace tn
