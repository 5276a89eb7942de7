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
// modes[(a * 3 + d) * n + i] = (e_a x X_i)_d, three modes, FP64
int null_space_modes_raw(int64_t n, int nr, const double* coords, const double* radii, double* modes, cudaStream_t st);
// doubles of per-block partials penalty_apply needs
int penalty_partials_size();
// alpha_k = eps <src, mode_k>_owned, then dst += sum_k alpha_k mode_k (3 launches, alpha left on the device)
template <typename T>
int penalty_apply(int64_t n, int nr, const uint8_t* owned_lat, const T* const* src, T* const* dst, const T* modes,
                  double eps, double* partials, double* alpha, cudaStream_t st);
// a <-> b elementwise, ncomp components
template <typename T>
int swap_vectors(int64_t n, int ncomp, T* const* a, T* const* b, cudaStream_t st);

}  // namespace tn
