// Dense direct solve of the coarsest multigrid level (sm_100a, FP64).
//
// The coarsest operator of the hierarchy (level 2 of a level-6 shell: 810 unique nodes, 2430 unknowns) is small
// enough to invert once at set-up. Its assembled matrix is built column by column by applying the stored
// (boundary-baked) coarse operator to unit vectors that hold 1 on every interface copy of one unknown, then
// inverted in place by Gauss-Jordan elimination without pivoting (the matrix is symmetric positive definite:
// Dirichlet rows keep their diagonal). Each V-cycle then solves exactly with one dense matrix-vector product,
// instead of the reference's 50 preconditioner-free CG iterations (pcg.hpp:81-169, stokes_solver.hpp:469);
// this is the `dense` coarse option of the solver interface.
//
// Unknown numbering: unknown (c, u) = c * nu + u for component c and unique node u, u running over the owned
// copies in storage order; uid[i] maps every stored node (all copies) to its unique node, rep[u] to the owned
// copy. The solve gathers the right-hand side at rep[], multiplies, and scatters the result to every copy, so
// x leaves consistent (all copies equal), as the CG solution does.
#include <algorithm>
#include <cstdint>

#include "tn_kernels.hpp"

namespace tn {
namespace {

constexpr int kThreads = 256;

__global__ void unit_fill_kernel(int64_t nodes, int64_t stride, int nu, const int32_t* __restrict__ uid, int dof,
                                 double* __restrict__ v)
{
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= nodes) return;
    const int u = uid[i];
#pragma unroll
    for (int c = 0; c < 3; ++c) v[c * stride + i] = (c * nu + u == dof) ? 1.0 : 0.0;
}

// K[row][col] = y at the owned copy of row's unknown
__global__ void column_gather_kernel(int nu, int64_t stride, const int32_t* __restrict__ rep,
                                     const double* __restrict__ y, int col, int64_t nd, double* __restrict__ K)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= 3 * nu) return;
    const int c = r / nu, u = r - c * nu;
    K[static_cast<int64_t>(r) * nd + col] = y[c * stride + rep[u]];
}

// Gauss-Jordan step k (in place, no pivoting): colk = column k (old values) ...
__global__ void gj_save_column_kernel(int64_t n, int k, const double* __restrict__ A, double* __restrict__ colk)
{
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i < n) colk[i] = A[i * n + k];
}
// ... row k scaled by 1 / pivot with its pivot entry replaced by 1 first ...
__global__ void gj_row_kernel(int64_t n, int k, double* __restrict__ A, const double* __restrict__ colk)
{
    const int64_t j = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (j >= n) return;
    const double pinv = 1.0 / colk[k];
    A[k * n + j]      = (j == k ? 1.0 : A[k * n + j]) * pinv;
}
// ... then every other row i: A[i][j] = (j == k ? 0 : A[i][j]) - colk[i] * A[k][j]
__global__ void gj_eliminate_kernel(int64_t n, int k, double* __restrict__ A, const double* __restrict__ colk)
{
    const int64_t i = blockIdx.y;
    if (i == k) return;
    const double f = colk[i];
    for (int64_t j = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; j < n;
         j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const double a   = (j == k) ? 0.0 : A[i * n + j];
        A[i * n + j]     = a - f * A[k * n + j];
    }
}

// y = Kinv b_u: each CTA stages the gathered right-hand side in shared memory; one warp per row
__global__ void __launch_bounds__(kThreads) dense_gemv_kernel(int nu, int64_t stride, const int32_t* __restrict__ rep,
                                                              const double* __restrict__ Kinv,
                                                              const double* __restrict__ b, double* __restrict__ y)
{
    extern __shared__ double bu[];
    const int nd = 3 * nu;
    for (int r = threadIdx.x; r < nd; r += blockDim.x) {
        const int c = r / nu, u = r - c * nu;
        bu[r]       = b[c * stride + rep[u]];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int warps_total = gridDim.x * (blockDim.x >> 5);
    for (int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); row < nd; row += warps_total) {
        const double* K = Kinv + static_cast<int64_t>(row) * nd;
        double        s = 0.0;
        for (int j = lane; j < nd; j += 32) s = fma(K[j], bu[j], s);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) y[row] = s;
    }
}

__global__ void scatter_kernel(int64_t nodes, int64_t stride, int nu, const int32_t* __restrict__ uid,
                               const double* __restrict__ y, double* __restrict__ x)
{
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= nodes) return;
    const int u = uid[i];
#pragma unroll
    for (int c = 0; c < 3; ++c) x[c * stride + i] = y[c * nu + u];
}

inline unsigned blocks_for(int64_t n) { return static_cast<unsigned>((n + kThreads - 1) / kThreads); }
inline int      status(int launches)
{
    note_launch(launches);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace

int dense_unit_vector(int64_t nodes, int64_t stride, int nu, const int32_t* uid, int dof, double* v, cudaStream_t st)
{
    unit_fill_kernel<<<blocks_for(nodes), kThreads, 0, st>>>(nodes, stride, nu, uid, dof, v);
    return status(1);
}

int dense_gather_column(int nu, int64_t stride, const int32_t* rep, const double* y, int col, double* K,
                        cudaStream_t st)
{
    const int64_t nd = 3 * static_cast<int64_t>(nu);
    column_gather_kernel<<<blocks_for(nd), kThreads, 0, st>>>(nu, stride, rep, y, col, nd, K);
    return status(1);
}

int dense_invert_spd(int64_t n, double* A, double* colk, cudaStream_t st)
{
    const unsigned gx = static_cast<unsigned>(std::min<int64_t>((n + kThreads - 1) / kThreads, 16));
    for (int k = 0; k < n; ++k) {
        gj_save_column_kernel<<<blocks_for(n), kThreads, 0, st>>>(n, k, A, colk);
        gj_row_kernel<<<blocks_for(n), kThreads, 0, st>>>(n, k, A, colk);
        gj_eliminate_kernel<<<dim3(gx, static_cast<unsigned>(n)), kThreads, 0, st>>>(n, k, A, colk);
        if (cudaGetLastError() != cudaSuccess) return -1;
    }
    return status(3 * static_cast<int>(n));
}

int dense_coarse_prepare(int unknowns)
{
    if (unknowns > kDenseCoarseMaxUnknowns) return -2;
    // The limit is raised to the largest supported system, not to this one:
    // a smaller solver prepared later must not lower it under a larger one.
    const size_t smem = sizeof(double) * static_cast<size_t>(kDenseCoarseMaxUnknowns);
    return cudaFuncSetAttribute(dense_gemv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(smem)) == cudaSuccess
               ? 0
               : -1;
}

int dense_coarse_solve(int64_t nodes, int64_t stride, int nu, const int32_t* uid, const int32_t* rep,
                       const double* Kinv, const double* b, double* y, double* x, cudaStream_t st)
{
    const int    nd   = 3 * nu;
    const size_t smem = sizeof(double) * static_cast<size_t>(nd);
    if (nd > kDenseCoarseMaxUnknowns) return -2;
    const unsigned rows_per_cta = kThreads / 32;
    const unsigned ctas         = static_cast<unsigned>((nd + rows_per_cta - 1) / rows_per_cta);
    dense_gemv_kernel<<<ctas, kThreads, smem, st>>>(nu, stride, rep, Kinv, b, y);
    scatter_kernel<<<blocks_for(nodes), kThreads, 0, st>>>(nodes, stride, nu, uid, y, x);
    return status(2);
}

}  // namespace tn
