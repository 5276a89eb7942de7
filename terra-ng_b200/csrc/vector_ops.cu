// Nodal-vector kernels: interface sum over diamond-edge duplicates, fused
// multi-component BLAS-1 and owned-node reductions (FP64 and FP32).
//
// The reference runs one Kokkos launch per component and per neighbour pair
// (kernels/common/grid_operations.hpp:132-346, communication_plan.hpp:471-517);
// here each operation is one launch over all components, and the interface
// sum is one gather-sum launch over the precomputed duplicate classes.
#include <algorithm>

#include "tn_device.cuh"
#include "tn_kernels.hpp"

namespace tn {
namespace {

constexpr int kMaxComp = 4;

template <typename T>
struct Comps {
    T* p[kMaxComp];
};
template <typename T>
struct CComps {
    const T* p[kMaxComp];
};

// ---------------------------------------------------------------------------
// Interface sum: every member of a duplicate class receives the class sum.
// One thread per (class, r, component); members are read along r (coalesced).
// A class has at most 5 members (the poles); their values are loaded before
// the sum so the loads overlap, and summed in member order.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void iface_kernel(int num_classes, const int32_t* __restrict__ off, const int32_t* __restrict__ mem, int nr,
                             int ncomp, Comps<T> v)
{
    const int cls = blockIdx.x;
    const int c   = blockIdx.z;
    const int r   = blockIdx.y * blockDim.x + threadIdx.x;
    if (cls >= num_classes || r >= nr || c >= ncomp) return;
    const int b = __ldg(off + cls), e = __ldg(off + cls + 1);
    T*        p = v.p[c];
    constexpr int kMax = 8;
    if (e - b <= kMax) {
        int64_t idx[kMax];
        T       val[kMax];
#pragma unroll
        for (int k = 0; k < kMax; ++k)
            if (b + k < e) idx[k] = static_cast<int64_t>(__ldg(mem + b + k)) * nr + r;
#pragma unroll
        for (int k = 0; k < kMax; ++k)
            if (b + k < e) val[k] = p[idx[k]];
        T s = T(0);
#pragma unroll
        for (int k = 0; k < kMax; ++k)
            if (b + k < e) s += val[k];
#pragma unroll
        for (int k = 0; k < kMax; ++k)
            if (b + k < e) p[idx[k]] = s;
    } else {
        T s = T(0);
        for (int m = b; m < e; ++m) s += p[static_cast<int64_t>(mem[m]) * nr + r];
        for (int m = b; m < e; ++m) p[static_cast<int64_t>(mem[m]) * nr + r] = s;
    }
}

template <typename T, int NT>
__global__ void lincomb_kernel(int64_t n, int ncomp, Comps<T> y, T c0, T ca, T cb, T cc, CComps<T> x0, CComps<T> x1,
                               CComps<T> x2)
{
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    for (int c = 0; c < ncomp; ++c) {
        T*       yc  = y.p[c];
        const T* a   = x0.p[c];
        const T* b   = x1.p[c];
        const T* cc_ = x2.p[c];
        for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
            T v = c0;
            if (NT >= 1) v += ca * a[i];
            if (NT >= 2) v += cb * b[i];
            if (NT >= 3) v += cc * cc_[i];
            yc[i] = v;
        }
    }
}

template <typename T>
__global__ void scale_kernel(int64_t n, int ncomp, Comps<T> y, CComps<T> x)
{
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    for (int c = 0; c < ncomp; ++c)
        for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
            y.p[c][i] *= x.p[c][i];
}

template <typename T>
__global__ void invert_kernel(int64_t n, int ncomp, Comps<T> y)
{
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    for (int c = 0; c < ncomp; ++c)
        for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
            y.p[c][i] = T(1) / y.p[c][i];
}

__device__ __forceinline__ double warp_sum(double v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v)
{
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

constexpr int kRedBlocks  = 592;  // 4 x 148 SMs
constexpr int kRedThreads = 256;

// Owned-masked dot accumulated in double; fixed grid => deterministic order.
template <typename T>
__global__ void __launch_bounds__(kRedThreads) dot_partial_kernel(int64_t n, int nr, int ncomp,
                                                                   const uint8_t* __restrict__ owned, CComps<T> a,
                                                                   CComps<T> b, double* partials)
{
    __shared__ double red[kRedThreads / 32];
    double            acc    = 0.0;
    const int64_t     stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    const uint32_t    unr    = static_cast<uint32_t>(nr);
    for (int c = 0; c < ncomp; ++c) {
        const T* __restrict__ pa = a.p[c];
        const T* __restrict__ pb = b.p[c];
        for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
            const int64_t lat = (n < 0xffffffffll) ? static_cast<int64_t>(static_cast<uint32_t>(i) / unr) : i / nr;
            if (owned[lat]) acc += static_cast<double>(pa[i]) * static_cast<double>(pb[i]);
        }
    }
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < kRedThreads / 32 ? red[threadIdx.x] : 0.0;
        v        = warp_sum(v);
        if (threadIdx.x == 0) partials[blockIdx.x] = v;
    }
}

__global__ void finish_sum_kernel(const double* partials, int np, double* out)
{
    __shared__ double red[32];
    double            acc = 0.0;
    for (int i = threadIdx.x; i < np; i += blockDim.x) acc += partials[i];
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        v        = warp_sum(v);
        if (threadIdx.x == 0) *out = v;
    }
}

template <typename T>
__global__ void __launch_bounds__(kRedThreads) maxabs_kernel(int64_t n, int ncomp, CComps<T> a, double* partials,
                                                              int* nanflag)
{
    __shared__ double red[kRedThreads / 32];
    double            m      = 0.0;
    bool              bad    = false;
    const int64_t     stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    for (int c = 0; c < ncomp; ++c)
        for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
            const double v = static_cast<double>(a.p[c][i]);
            if (!isfinite(v)) bad = true;
            m = fmax(m, fabs(v));
        }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicExch(nanflag, 1);
    m = warp_max(m);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < kRedThreads / 32 ? red[threadIdx.x] : 0.0;
        v        = warp_max(v);
        if (threadIdx.x == 0) partials[blockIdx.x] = v;
    }
}

__global__ void finish_max_kernel(const double* partials, int np, double* out)
{
    double m = 0.0;
    for (int i = threadIdx.x; i < np; i += blockDim.x) m = fmax(m, partials[i]);
    m = warp_max(m);
    if (threadIdx.x == 0) *out = m;
}

__global__ void f64_to_f32_kernel(int64_t n, const double* in, float* out)
{
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        out[i] = static_cast<float>(in[i]);
}
__global__ void f32_to_f64_kernel(int64_t n, const float* in, double* out)
{
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        out[i] = static_cast<double>(in[i]);
}

inline int grid_for(int64_t n, int threads)
{
    int64_t b = (n + threads - 1) / threads;
    if (b > 148 * 16) b = 148 * 16;
    if (b < 1) b = 1;
    return static_cast<int>(b);
}

inline int launch_status(int kernels = 1)
{
    note_launch(kernels);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

}  // namespace

template <typename T>
int interface_sum(const IfaceTable& t, int nr, int ncomp, T* const* comps, cudaStream_t stream)
{
    if (ncomp > kMaxComp || ncomp < 1) return -1;
    if (t.num_classes == 0) return 0;
    Comps<T> v{};
    for (int c = 0; c < ncomp; ++c) v.p[c] = comps[c];
    const int threads = std::min(256, (nr + 31) / 32 * 32);
    dim3      grid(t.num_classes, (nr + threads - 1) / threads, ncomp);
    iface_kernel<T><<<grid, threads, 0, stream>>>(t.num_classes, t.offset, t.members, nr, ncomp, v);
    return launch_status();
}

template <typename T>
int lincomb(int64_t n, int ncomp, T* const* y, T c0, int nterms, const T* c, const T* const* x0, const T* const* x1,
            const T* const* x2, cudaStream_t stream)
{
    if (ncomp > kMaxComp || ncomp < 1 || nterms < 0 || nterms > 3) return -1;
    Comps<T>  yy{};
    CComps<T> a{}, b{}, cc{};
    for (int k = 0; k < ncomp; ++k) {
        yy.p[k] = y[k];
        a.p[k]  = nterms >= 1 ? x0[k] : nullptr;
        b.p[k]  = nterms >= 2 ? x1[k] : nullptr;
        cc.p[k] = nterms >= 3 ? x2[k] : nullptr;
    }
    const T   ca = nterms >= 1 ? c[0] : T(0), cb = nterms >= 2 ? c[1] : T(0), c3 = nterms >= 3 ? c[2] : T(0);
    const int g  = grid_for(n, 256);
    switch (nterms) {
    case 0: lincomb_kernel<T, 0><<<g, 256, 0, stream>>>(n, ncomp, yy, c0, ca, cb, c3, a, b, cc); break;
    case 1: lincomb_kernel<T, 1><<<g, 256, 0, stream>>>(n, ncomp, yy, c0, ca, cb, c3, a, b, cc); break;
    case 2: lincomb_kernel<T, 2><<<g, 256, 0, stream>>>(n, ncomp, yy, c0, ca, cb, c3, a, b, cc); break;
    default: lincomb_kernel<T, 3><<<g, 256, 0, stream>>>(n, ncomp, yy, c0, ca, cb, c3, a, b, cc); break;
    }
    return launch_status();
}

template <typename T>
int scale_inplace(int64_t n, int ncomp, T* const* y, const T* const* x, cudaStream_t stream)
{
    if (ncomp > kMaxComp || ncomp < 1) return -1;
    Comps<T>  yy{};
    CComps<T> xx{};
    for (int k = 0; k < ncomp; ++k) {
        yy.p[k] = y[k];
        xx.p[k] = x[k];
    }
    scale_kernel<T><<<grid_for(n, 256), 256, 0, stream>>>(n, ncomp, yy, xx);
    return launch_status();
}

template <typename T>
int invert_inplace(int64_t n, int ncomp, T* const* y, cudaStream_t stream)
{
    if (ncomp > kMaxComp || ncomp < 1) return -1;
    Comps<T> yy{};
    for (int k = 0; k < ncomp; ++k) yy.p[k] = y[k];
    invert_kernel<T><<<grid_for(n, 256), 256, 0, stream>>>(n, ncomp, yy);
    return launch_status();
}

template <typename T>
int masked_dot(int64_t n, int nr, int ncomp, const uint8_t* owned_lat, const T* const* a, const T* const* b,
               double* out_dev, double* partials, cudaStream_t stream)
{
    if (ncomp > kMaxComp || ncomp < 1) return -1;
    CComps<T> aa{}, bb{};
    for (int k = 0; k < ncomp; ++k) {
        aa.p[k] = a[k];
        bb.p[k] = b[k];
    }
    dot_partial_kernel<T><<<kRedBlocks, kRedThreads, 0, stream>>>(n, nr, ncomp, owned_lat, aa, bb, partials);
    finish_sum_kernel<<<1, 1024, 0, stream>>>(partials, kRedBlocks, out_dev);
    return launch_status(2);
}

template <typename T>
int max_abs_and_nan(int64_t n, int ncomp, const T* const* a, double* out_dev, int* nan_dev, cudaStream_t stream)
{
    if (ncomp > kMaxComp || ncomp < 1) return -1;
    CComps<T> aa{};
    for (int k = 0; k < ncomp; ++k) aa.p[k] = a[k];
    // partial maxima go to out_dev[1 .. kRedBlocks]
    maxabs_kernel<T><<<kRedBlocks, kRedThreads, 0, stream>>>(n, ncomp, aa, out_dev + 1, nan_dev);
    finish_max_kernel<<<1, 32, 0, stream>>>(out_dev + 1, kRedBlocks, out_dev);
    return launch_status(2);
}

int convert_f64_to_f32(int64_t n, const double* in, float* out, cudaStream_t stream)
{
    f64_to_f32_kernel<<<grid_for(n, 256), 256, 0, stream>>>(n, in, out);
    return launch_status();
}
int convert_f32_to_f64(int64_t n, const float* in, double* out, cudaStream_t stream)
{
    f32_to_f64_kernel<<<grid_for(n, 256), 256, 0, stream>>>(n, in, out);
    return launch_status();
}

#define TN_INST(T)                                                                                                  \
    template int interface_sum<T>(const IfaceTable&, int, int, T* const*, cudaStream_t);                           \
    template int lincomb<T>(int64_t, int, T* const*, T, int, const T*, const T* const*, const T* const*,          \
                            const T* const*, cudaStream_t);                                                         \
    template int scale_inplace<T>(int64_t, int, T* const*, const T* const*, cudaStream_t);                         \
    template int invert_inplace<T>(int64_t, int, T* const*, cudaStream_t);                                         \
    template int masked_dot<T>(int64_t, int, int, const uint8_t*, const T* const*, const T* const*, double*,       \
                               double*, cudaStream_t);                                                              \
    template int max_abs_and_nan<T>(int64_t, int, const T* const*, double*, int*, cudaStream_t);
TN_INST(double)
TN_INST(float)
#undef TN_INST

int reduction_partials_size() { return kRedBlocks + 1; }

}  // namespace tn
