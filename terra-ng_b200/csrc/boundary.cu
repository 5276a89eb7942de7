// Boundary treatment of nodal vectors and the free-slip/free-slip null-space penalty (sm_100a).
//
// * assign_masked: strong Dirichlet on a right-hand side, dst = m value + (1 - m) dst with m = 1 where the
//   node's boundary flags contain `flag` (kernels/common/grid_operations.hpp:54-131, util/bit_masking.hpp:43-53).
// * freeslip_project / rotate_nt: the normal-tangential rotation of free-slip nodes
//   (linalg/trafo/local_basis_trafo_normal_tangential.hpp:34-186) and the right-hand-side projection built on
//   it (fe/strong_algebraic_freeslip_enforcement.hpp:22-38): rotate, zero the normal part, rotate back.
// * penalty_*: the three rotation modes e_i x X of a shell with free slip on both boundaries, orthonormalised
//   with owned-node dots, and the penalty dst += eps sum_i (n_i^T src) n_i added on every interface copy before
//   the interface sum (epsilon_divdiv_kerngen.hpp:324-445, :711-785). The orthonormal modes are a fixed 3 x 3
//   combination C of the raw ones (from their Gram matrix), so the kernels evaluate the raw modes from the
//   coordinates and apply C to three dots instead of streaming nine stored mode arrays.
//
// Node flags follow from the radial index alone (grid/shell/bit_masks.hpp:82-136): CMB on r = 0, SURFACE on
// r = nr - 1, INNER elsewhere, so no mask array is read. All kernels are flat grids over (10, nl, nl, nr) with r
// fastest; the penalty dots reduce in a fixed order (per-block partials, then one block), so results are
// reproducible run to run.
#include <algorithm>
#include <cstdint>

#include "tn_boundary.hpp"
#include "tn_kernels.hpp"

namespace tn {
namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ int shell_flag(int r, int nr)
{
    return r == 0 ? kFlagCMB : (r == nr - 1 ? kFlagSurface : kFlagInner);
}

__device__ __forceinline__ bool has_flag(int mask, int flag)
{
    return flag == 0 ? mask == 0 : (mask & flag) == flag;
}

// Rows (n, t1, t2) of the rotation into the normal-tangential basis of the unit normal direction c
// (trafo_mat_cartesian_to_normal_tangential): n = c / |c|; the reference axis is the coordinate axis least
// aligned with n (x on ties with y or z, then y); t1 = (ref x n) / |ref x n|; t2 = (n x t1) / |n x t1|.
// Vectors shorter than 1e-15 are left unnormalised, as dense::Vec::normalize does.
template <typename T>
__device__ __forceinline__ void normalize3(T v[3])
{
    const T mag = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    if (mag > T(1e-15)) {
        v[0] /= mag;
        v[1] /= mag;
        v[2] /= mag;
    }
}
template <typename T>
__device__ __forceinline__ void cross3(const T a[3], const T b[3], T o[3])
{
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}
template <typename T>
__device__ void nt_basis(const T c[3], T R[3][3])
{
    T n[3] = {c[0], c[1], c[2]};
    normalize3(n);
    const T ax = fabs(n[0]), ay = fabs(n[1]), az = fabs(n[2]);
    T       ref[3] = {T(0), T(0), T(0)};
    if (ax <= ay && ax <= az)
        ref[0] = T(1);
    else if (ay <= ax && ay <= az)
        ref[1] = T(1);
    else
        ref[2] = T(1);
    T t1[3];
    cross3(ref, n, t1);
    normalize3(t1);
    const T eps = sizeof(T) == 8 ? T(1e-15) : T(1e-6);
    if (sqrt(t1[0] * t1[0] + t1[1] * t1[1] + t1[2] * t1[2]) < eps) {
        t1[0] = n[1];
        t1[1] = -n[0];
        t1[2] = T(0);
        normalize3(t1);
    }
    T t2[3];
    cross3(n, t1, t2);
    normalize3(t2);
    for (int j = 0; j < 3; ++j) {
        R[0][j] = n[j];
        R[1][j] = t1[j];
        R[2][j] = t2[j];
    }
}

template <typename T>
__global__ void assign_masked_kernel(int64_t n, int nr, int ncomp, Ptrs4<T> v, int flag, T value)
{
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const T m = has_flag(shell_flag(static_cast<int>(i % nr), nr), flag) ? T(1) : T(0);
    for (int c = 0; c < ncomp; ++c) v.p[c][i] = m * value + (T(1) - m) * v.p[c][i];
}

// mode 0: cartesian -> (n, t1, t2); 1: back; 2: both with the normal component zeroed in between
template <typename T>
__global__ void rotate_kernel(int64_t n, int nr, const T* __restrict__ coords, Ptrs4<T> v, int flag, int mode)
{
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    if (!has_flag(shell_flag(static_cast<int>(i % nr), nr), flag)) return;
    const int64_t col  = i / nr;
    const T       c[3] = {coords[3 * col], coords[3 * col + 1], coords[3 * col + 2]};
    T             R[3][3];
    nt_basis(c, R);
    T x[3] = {v.p[0][i], v.p[1][i], v.p[2][i]};
    T y[3];
    if (mode != 1) {
        for (int a = 0; a < 3; ++a) y[a] = R[a][0] * x[0] + R[a][1] * x[1] + R[a][2] * x[2];
        if (mode == 0) {
            for (int a = 0; a < 3; ++a) v.p[a][i] = y[a];
            return;
        }
        y[0] = T(0);  // assign_masked on the normal component: 1 * 0 + 0 * y0
        for (int a = 0; a < 3; ++a) x[a] = y[a];
    }
    for (int a = 0; a < 3; ++a) y[a] = R[0][a] * x[0] + R[1][a] * x[1] + R[2][a] * x[2];
    for (int a = 0; a < 3; ++a) v.p[a][i] = y[a];
}

// Raw rotation modes at node i: mode a holds e_a x X (X = unit coordinate times radius). The reference's free-slip
// pass over them selects nodes flagged CMB | SURFACE together, which no node is, so it changes nothing and is
// not repeated here. The modes are evaluated where they are used, from the coordinates and radii (24 bytes per
// lateral column and 8 per radius), instead of being stored as nine arrays.
template <typename T>
__device__ __forceinline__ void raw_modes(const T* __restrict__ coords, const T* __restrict__ radii, int col, int r,
                                          T (&m)[3][3])
{
    const T R    = radii[r];
    const T X[3] = {coords[3 * col] * R, coords[3 * col + 1] * R, coords[3 * col + 2] * R};
#pragma unroll
    for (int axis = 0; axis < 3; ++axis) {
        const int a1 = (axis + 1) % 3, a2 = (axis + 2) % 3;
        m[axis][axis] = T(0);
        m[axis][a1]   = X[a2];
        m[axis][a2]   = -X[a1];
    }
}

// block sums of NV values, written to partials[blockIdx.x * NV + k]
template <int NV>
__device__ __forceinline__ void block_partials(double (&s)[NV], double* __restrict__ partials)
{
    __shared__ double red[NV][kThreads / 32];
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double v = s[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) red[k][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x < NV) {
        double v = 0.0;
        for (int w = 0; w < kThreads / 32; ++w) v += red[threadIdx.x][w];
        partials[blockIdx.x * NV + threadIdx.x] = v;
    }
}

// per-block partial sums of the owned-node Gram matrix <m_a, m_b> of the raw modes (a <= b: 00 01 02 11 12 22)
__global__ void penalty_gram_kernel(int n, int nr, const uint8_t* __restrict__ owned_lat,
                                    const double* __restrict__ coords, const double* __restrict__ radii,
                                    double* __restrict__ partials)
{
    double s[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int col = i / nr;
        if (!owned_lat[col]) continue;
        double m[3][3];
        raw_modes<double>(coords, radii, col, i - col * nr, m);
        int k = 0;
        for (int a = 0; a < 3; ++a)
            for (int b = a; b < 3; ++b, ++k) s[k] += m[a][0] * m[b][0] + m[a][1] * m[b][1] + m[a][2] * m[b][2];
    }
    block_partials<6>(s, partials);
}

// per-block partial sums of the owned-node dots <src, m_a> with the raw modes
template <typename T>
__global__ void penalty_dots_kernel(int n, int nr, const uint8_t* __restrict__ owned_lat, const T* __restrict__ coords,
                                    const T* __restrict__ radii, Ptrs4<const T> src, double* __restrict__ partials)
{
    double s[3] = {0.0, 0.0, 0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int col = i / nr;
        if (!owned_lat[col]) continue;
        T m[3][3];
        raw_modes<T>(coords, radii, col, i - col * nr, m);
        const double sv[3] = {static_cast<double>(src.p[0][i]), static_cast<double>(src.p[1][i]),
                              static_cast<double>(src.p[2][i])};
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int d = 0; d < 3; ++d) s[a] += static_cast<double>(m[a][d]) * sv[d];
    }
    block_partials<3>(s, partials);
}

// sum the block partials (NV values per block) in a fixed order into out[0 .. NV-1]
template <int NV>
__device__ __forceinline__ void sum_partials(int nblocks, const double* __restrict__ partials, double (&out)[NV])
{
    __shared__ double red[NV][kThreads];
    for (int k = 0; k < NV; ++k) {
        double v = 0.0;
        for (int b = threadIdx.x; b < nblocks; b += kThreads) v += partials[b * NV + k];
        red[k][threadIdx.x] = v;
    }
    __syncthreads();
    for (int st = kThreads / 2; st > 0; st >>= 1) {
        if (threadIdx.x < st)
            for (int k = 0; k < NV; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + st];
        __syncthreads();
    }
    for (int k = 0; k < NV; ++k) out[k] = red[k][0];
}

__global__ void gram_finish_kernel(int nblocks, const double* __restrict__ partials, double* __restrict__ gram)
{
    double g[6];
    sum_partials<6>(nblocks, partials, g);
    if (threadIdx.x < 6) gram[threadIdx.x] = g[threadIdx.x];
}

// With the orthonormal modes n_i = sum_a C[i][a] m_a: dot_i = <src, n_i> = sum_a C[i][a] r_a, and the penalty
// eps sum_i dot_i n_i = sum_a beta_a m_a with beta_a = eps sum_i C[i][a] dot_i.
__global__ void penalty_finish_kernel(int nblocks, const double* __restrict__ partials, PenaltyCoef coef, double eps,
                                      double* __restrict__ beta)
{
    double r[3];
    sum_partials<3>(nblocks, partials, r);
    if (threadIdx.x == 0) {
        double dot[3];
        for (int i = 0; i < 3; ++i)
            dot[i] = coef.c[3 * i] * r[0] + coef.c[3 * i + 1] * r[1] + coef.c[3 * i + 2] * r[2];
        for (int a = 0; a < 3; ++a)
            beta[a] = eps * (coef.c[a] * dot[0] + coef.c[3 + a] * dot[1] + coef.c[6 + a] * dot[2]);
    }
}

template <typename T>
__global__ void penalty_axpy_kernel(int n, int nr, const T* __restrict__ coords, const T* __restrict__ radii,
                                    Ptrs4<T> dst, const double* __restrict__ beta)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int col = i / nr;
    T         m[3][3];
    raw_modes<T>(coords, radii, col, i - col * nr, m);
    const T b0 = static_cast<T>(beta[0]), b1 = static_cast<T>(beta[1]), b2 = static_cast<T>(beta[2]);
#pragma unroll
    for (int d = 0; d < 3; ++d) dst.p[d][i] += b0 * m[0][d] + b1 * m[1][d] + b2 * m[2][d];
}

template <typename T>
__global__ void swap_kernel(int64_t n, Ptrs4<T> a, Ptrs4<T> b, int ncomp)
{
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    for (int c = 0; c < ncomp; ++c) {
        const T t = a.p[c][i];
        a.p[c][i] = b.p[c][i];
        b.p[c][i] = t;
    }
}

inline unsigned blocks_for(int64_t n) { return static_cast<unsigned>((n + kThreads - 1) / kThreads); }

}  // namespace

template <typename T>
int assign_masked(int64_t n, int nr, int ncomp, T* const* v, int flag, T value, cudaStream_t st)
{
    if (n == 0) return 0;
    Ptrs4<T> p;
    for (int c = 0; c < ncomp; ++c) p.p[c] = v[c];
    assign_masked_kernel<T><<<blocks_for(n), kThreads, 0, st>>>(n, nr, ncomp, p, flag, value);
    note_launch();
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

template <typename T>
int rotate_normal_tangential(int64_t n, int nr, const T* coords, T* const* v, int flag, int mode, cudaStream_t st)
{
    if (n == 0) return 0;
    Ptrs4<T> p;
    for (int c = 0; c < 3; ++c) p.p[c] = v[c];
    rotate_kernel<T><<<blocks_for(n), kThreads, 0, st>>>(n, nr, coords, p, flag, mode);
    note_launch();
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int penalty_partials_size() { return 6 * kPenaltyBlocks; }

int penalty_gram(int64_t n, int nr, const uint8_t* owned_lat, const double* coords, const double* radii,
                 double* partials, double* gram, cudaStream_t st)
{
    if (n >= (int64_t(1) << 31)) return -1;
    const int nb = static_cast<int>(std::min<int64_t>(kPenaltyBlocks, (n + kThreads - 1) / kThreads));
    penalty_gram_kernel<<<nb, kThreads, 0, st>>>(static_cast<int>(n), nr, owned_lat, coords, radii, partials);
    gram_finish_kernel<<<1, kThreads, 0, st>>>(nb, partials, gram);
    note_launch(2);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

template <typename T>
int penalty_apply(int64_t n, int nr, const uint8_t* owned_lat, const T* coords, const T* radii, const T* const* src,
                  T* const* dst, const PenaltyCoef& coef, double eps, double* partials, double* beta, cudaStream_t st)
{
    if (n >= (int64_t(1) << 31)) return -1;
    Ptrs4<const T> s;
    Ptrs4<T>       d;
    for (int c = 0; c < 3; ++c) {
        s.p[c] = src[c];
        d.p[c] = dst[c];
    }
    const int ni = static_cast<int>(n);
    const int nb = static_cast<int>(std::min<int64_t>(kPenaltyBlocks, (n + kThreads - 1) / kThreads));
    penalty_dots_kernel<T><<<nb, kThreads, 0, st>>>(ni, nr, owned_lat, coords, radii, s, partials);
    penalty_finish_kernel<<<1, kThreads, 0, st>>>(nb, partials, coef, eps, beta);
    penalty_axpy_kernel<T><<<blocks_for(n), kThreads, 0, st>>>(ni, nr, coords, radii, d, beta);
    note_launch(3);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

template <typename T>
int swap_vectors(int64_t n, int ncomp, T* const* a, T* const* b, cudaStream_t st)
{
    if (n == 0) return 0;
    Ptrs4<T> pa, pb;
    for (int c = 0; c < ncomp; ++c) {
        pa.p[c] = a[c];
        pb.p[c] = b[c];
    }
    swap_kernel<T><<<blocks_for(n), kThreads, 0, st>>>(n, pa, pb, ncomp);
    note_launch();
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

template int assign_masked<double>(int64_t, int, int, double* const*, int, double, cudaStream_t);
template int assign_masked<float>(int64_t, int, int, float* const*, int, float, cudaStream_t);
template int rotate_normal_tangential<double>(int64_t, int, const double*, double* const*, int, int, cudaStream_t);
template int rotate_normal_tangential<float>(int64_t, int, const float*, float* const*, int, int, cudaStream_t);
template int penalty_apply<double>(int64_t, int, const uint8_t*, const double*, const double*, const double* const*,
                                   double* const*, const PenaltyCoef&, double, double*, double*, cudaStream_t);
template int penalty_apply<float>(int64_t, int, const uint8_t*, const float*, const float*, const float* const*,
                                  float* const*, const PenaltyCoef&, double, double*, double*, cudaStream_t);
template int swap_vectors<double>(int64_t, int, double* const*, double* const*, cudaStream_t);
template int swap_vectors<float>(int64_t, int, float* const*, float* const*, cudaStream_t);

}  // namespace tn
