// Host-callable launchers of the sm_100a kernels. All pointers are device
// pointers; every launcher is asynchronous on `stream` and returns 0 or a
// negative launch error.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace tn {

// ----------------------------------------------------------------------------
// epsilon-div-div apply (epsdivdiv.cu)
// ----------------------------------------------------------------------------
template <typename T>
struct EddLaunch {
    int      nl = 0, nr = 0;
    const T* coords = nullptr;  // (10, nl, nl, 3)
    const T* radii  = nullptr;  // (nr)
    const T* k      = nullptr;  // nodal coefficient (10, nl, nl, nr) or nullptr
    const T* kq0    = nullptr;  // cell coefficient (10, nl-1, nl-1, nr-1) or nullptr
    const T* src[3] = {nullptr, nullptr, nullptr};
    T*       dst[3] = {nullptr, nullptr, nullptr};
    int      bc_cmb = 1, bc_surf = 1;  // 0 Neumann, 1 Dirichlet, 2 free-slip
    bool     diagonal = false;
    int      add      = 0;  // 0: dst = A src (owned nodes written), 1: dst += A src
    int      tile_y = 0, chunk_x = 0;  // 0: defaults
    int*     err = nullptr;            // device error word (bounded waits)
};
template <typename T>
int epsdivdiv_apply(const EddLaunch<T>& p, cudaStream_t stream);

// ----------------------------------------------------------------------------
// Coupling blocks and mass matrices (stokes_coupling.cu). All accumulate into
// their outputs (callers zero them for Replace mode).
// ----------------------------------------------------------------------------
template <typename T>
struct CouplingLaunch {
    int      nl = 0, nr = 0;  // fine (velocity) level
    const T* coords = nullptr;
    const T* radii  = nullptr;
    int      bc_cmb = 1, bc_surf = 1;
    const T* u[3]     = {nullptr, nullptr, nullptr};  // divergence input
    T*       p_out    = nullptr;                      // divergence output (coarse)
    const T* p_in     = nullptr;                      // gradient input (coarse)
    T*       u_out[3] = {nullptr, nullptr, nullptr};  // gradient output
};
template <typename T>
int divergence_apply(const CouplingLaunch<T>& p, cudaStream_t stream);
template <typename T>
int gradient_apply(const CouplingLaunch<T>& p, cudaStream_t stream);
template <typename T>
int kmass_lumped_add(int nl, int nr, const T* coords, const T* radii, const T* k, T* diag, cudaStream_t stream);
template <typename T>
int vector_mass_add(int nl, int nr, const T* coords, const T* radii, const T* const* src, T* const* dst,
                    cudaStream_t stream);

// ----------------------------------------------------------------------------
// Constant-weight grid transfers (transfer.cu). Levels given by the fine grid.
// prolongate_add: fine += P coarse (gather per fine node).
// restrict_owned: coarse = sum over owned fine neighbours (weights of
//                 prolongation_constant_weight); the interface sum follows.
// ----------------------------------------------------------------------------
template <typename T>
int prolongate_add(int nlf, int nrf, int ncomp, const T* const* coarse, T* const* fine, cudaStream_t stream);
template <typename T>
int restrict_owned(int nlf, int nrf, int ncomp, const uint8_t* owned_lat_fine, const T* const* fine, T* const* coarse,
                   cudaStream_t stream);

// ----------------------------------------------------------------------------
// Interface sum over diamond-edge duplicates (vector_ops.cu).
// classes: offsets (num_classes + 1) into members (lateral indices).
// ----------------------------------------------------------------------------
struct IfaceTable {
    int            num_classes = 0;
    const int32_t* offset      = nullptr;
    const int32_t* members     = nullptr;
};
template <typename T>
int interface_sum(const IfaceTable& t, int nr, int ncomp, T* const* comps, cudaStream_t stream);

// ----------------------------------------------------------------------------
// BLAS-1 on nodal vectors of n elements per component (vector_ops.cu).
// ----------------------------------------------------------------------------
// y = c0 + sum_i c[i] * x_i  (0..3 terms), per component, ncomp components.
template <typename T>
int lincomb(int64_t n, int ncomp, T* const* y, T c0, int nterms, const T* c, const T* const* x0, const T* const* x1,
            const T* const* x2, cudaStream_t stream);
// y *= x elementwise
template <typename T>
int scale_inplace(int64_t n, int ncomp, T* const* y, const T* const* x, cudaStream_t stream);
// y = 1 / y
template <typename T>
int invert_inplace(int64_t n, int ncomp, T* const* y, cudaStream_t stream);
// out = sum over owned nodes and components of a * b, accumulated in double.
// owned_lat: (10, nl, nl) flags; the node's lateral index is i / nr.
template <typename T>
int masked_dot(int64_t n, int nr, int ncomp, const uint8_t* owned_lat, const T* const* a, const T* const* b,
               double* out_dev, double* partials, cudaStream_t stream);
// out = max |a| ; out_flags = 1 if any NaN/Inf
template <typename T>
int max_abs_and_nan(int64_t n, int ncomp, const T* const* a, double* out_dev, int* nan_dev, cudaStream_t stream);
// precision conversion
int convert_f64_to_f32(int64_t n, const double* in, float* out, cudaStream_t stream);
int convert_f32_to_f64(int64_t n, const float* in, double* out, cudaStream_t stream);

}  // namespace tn
