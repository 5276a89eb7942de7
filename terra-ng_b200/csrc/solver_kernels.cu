// Kernels of the Krylov / multigrid solver layer.
//
// * Owned-node dot products over (block) vectors laid out as segments of
//   components (velocity on level L, pressure on level L-1), reduced in a fixed
//   order by the last block to finish (no second launch, bitwise reproducible),
//   with the result left in device memory so that the host does not wait.
// * The FGMRES modified Gram-Schmidt step fused into one pass: w -= h_{i-1}
//   v_{i-1} followed by h_i = <w, v_i> (fgmres.hpp:230-240 does the same
//   arithmetic as two launches per basis vector, dot then lincomb).
// * The Chebyshev-Jacobi update d = alpha D^-1 (b - A x) + beta d, x += d in one
//   pass (chebyshev.hpp:102-176 uses four BLAS-1 launches per step).
// * The coarsest-grid CG (pcg.hpp:81-169, identity preconditioner) as a single
//   thread-block-cluster kernel over stored element matrices: the CTAs of one
//   cluster synchronise with the hardware cluster barrier, so the whole solve is
//   one launch.
#include <cfloat>
#include <map>
#include <mutex>
#include <tuple>

#include <cooperative_groups.h>

#include "tn_device.cuh"
#include "tn_kernels.hpp"

namespace tn {
namespace {
namespace cg = cooperative_groups;

constexpr int kThreads = 256;
constexpr int kBlocks  = 592;  // 4 x 148 SMs

__device__ __forceinline__ double warp_sum(double v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block sum, then the last block of the grid sums the per-block partials in
// index order and writes *out (sqrt of it when take_sqrt).
__device__ void block_finish(double v, RedScratch rs, double* out, int take_sqrt)
{
    __shared__ double red[kThreads / 32];
    __shared__ int    is_last;
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int k = 0; k < kThreads / 32; ++k) s += red[k];
        rs.partials[blockIdx.x] = s;
        __threadfence();
        const unsigned t = atomicAdd(rs.counter, 1u);
        is_last          = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (is_last) {
        __threadfence();
        double s = 0.0;
        for (int k = threadIdx.x; k < static_cast<int>(gridDim.x); k += blockDim.x) s += __ldcg(rs.partials + k);
        s = warp_sum(s);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
        __syncthreads();
        if (threadIdx.x == 0) {
            double tot = 0.0;
            for (int k = 0; k < kThreads / 32; ++k) tot += red[k];
            *out        = take_sqrt ? sqrt(tot) : tot;
            *rs.counter = 0u;
        }
    }
}

__device__ __forceinline__ uint32_t lat_of(int64_t i, uint64_t rdiv)
{
    return static_cast<uint32_t>((static_cast<uint64_t>(i) * rdiv) >> 40);
}

template <typename T>
__global__ void __launch_bounds__(kThreads) vdot_kernel(VecDesc L, const T* __restrict__ a, const T* __restrict__ b,
                                                         RedScratch rs, double* out, int take_sqrt)
{
    double        acc    = 0.0;
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    for (int s = 0; s < L.nseg; ++s) {
        const VecSeg S = L.seg[s];
        for (int c = 0; c < S.ncomp; ++c) {
            const T* pa = a + S.offset + c * S.stride;
            const T* pb = b + S.offset + c * S.stride;
            for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < S.n; i += stride)
                if (S.owned[lat_of(i, S.rdiv)]) acc += static_cast<double>(pa[i]) * static_cast<double>(pb[i]);
        }
    }
    block_finish(acc, rs, out, take_sqrt);
}

// L2 residency of the Gram-Schmidt target. One Arnoldi step reads and writes
// w once per basis vector; w (the level-6 Stokes vector is 69 MB) fits in the
// 126 MB L2 while the basis vectors stream past it. w is loaded and stored
// with an evict_last policy and the basis vectors with streaming loads, so
// each step reads the two basis vectors it uses (v_{i-1}, partly still in L2
// from the step before, and v_i) from DRAM, instead of those two plus w read
// and written. The last step of an Arnoldi iteration (the norm) stores w
// with evict_normal, which hands the lines back to ordinary replacement before
// the preconditioner runs.
__device__ __forceinline__ uint64_t l2_policy(bool keep)
{
    uint64_t p;
    if (keep)
        asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    else
        asm volatile("createpolicy.fractional.L2::evict_normal.b64 %0, 1.0;" : "=l"(p));
    return p;
}

__device__ __forceinline__ double2 ld_policy(const double2* a, uint64_t pol)
{
    double2 v;
    asm volatile("ld.global.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;" : "=d"(v.x), "=d"(v.y) : "l"(a), "l"(pol));
    return v;
}

__device__ __forceinline__ void st_policy(double2* a, double2 v, uint64_t pol)
{
    asm volatile("st.global.L2::cache_hint.v2.f64 [%0], {%1, %2}, %3;" ::"l"(a), "d"(v.x), "d"(v.y), "l"(pol)
                 : "memory");
}

// Gram-Schmidt step over pairs of entries (components start at multiples of
// 64 entries, so pairs are 16-byte aligned); the odd tail entry is handled
// by the thread that owns pair index n / 2. Each thread takes kMgsUnroll
// grid-strided pairs per trip and issues all their loads before the first
// store, so that enough bytes are in flight to cover DRAM latency; the pairs
// are accumulated in the same order as a one-pair loop would.
constexpr int kMgsUnroll = 2;

// kSub: subtract h v_sub from w first (every step but the first);
// kDot: dot with v_dot (every step but the last, which takes ||w||^2).
template <bool kSub, bool kDot>
__global__ void __launch_bounds__(kThreads) mgs_kernel(VecDesc L, double* __restrict__ w,
                                                        const double* __restrict__ vsub, const double* hsub,
                                                        const double* __restrict__ vdot, RedScratch rs, double* out,
                                                        int take_sqrt)
{
    const double   h      = kSub ? *hsub : 0.0;
    const uint64_t pol    = l2_policy(kDot);
    double         acc    = 0.0;
    const int64_t  stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    for (int s = 0; s < L.nseg; ++s) {
        const VecSeg  S  = L.seg[s];
        const int64_t np = S.n / 2;
        for (int c = 0; c < S.ncomp; ++c) {
            const int64_t  o  = S.offset + c * S.stride;
            double2*       w2 = reinterpret_cast<double2*>(w + o);
            const double2* s2 = reinterpret_cast<const double2*>(vsub + o);
            const double2* d2 = reinterpret_cast<const double2*>(vdot + o);
            for (int64_t k0 = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; k0 < np;
                 k0 += kMgsUnroll * stride) {
                double2 wv[kMgsUnroll], sv[kMgsUnroll], dv[kMgsUnroll];
#pragma unroll
                for (int u = 0; u < kMgsUnroll; ++u) {
                    const int64_t k = k0 + u * stride;
                    if (k < np) {
                        wv[u] = ld_policy(w2 + k, pol);
                        if constexpr (kSub) sv[u] = __ldcs(s2 + k);
                        if constexpr (kDot) dv[u] = __ldcs(d2 + k);
                    }
                }
#pragma unroll
                for (int u = 0; u < kMgsUnroll; ++u) {
                    const int64_t k = k0 + u * stride;
                    if (k < np) {
                        if constexpr (kSub) {
                            wv[u].x = wv[u].x - h * sv[u].x;
                            wv[u].y = wv[u].y - h * sv[u].y;
                            st_policy(w2 + k, wv[u], pol);
                        }
                        const double2 d = kDot ? dv[u] : wv[u];
                        if (S.owned[lat_of(2 * k, S.rdiv)]) acc += wv[u].x * d.x;
                        if (S.owned[lat_of(2 * k + 1, S.rdiv)]) acc += wv[u].y * d.y;
                    }
                }
            }
            if ((S.n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
                const int64_t i  = S.n - 1;
                double        wi = w[o + i];
                if constexpr (kSub) {
                    wi       = wi - h * vsub[o + i];
                    w[o + i] = wi;
                }
                if (S.owned[lat_of(i, S.rdiv)]) acc += wi * (kDot ? vdot[o + i] : wi);
            }
        }
    }
    block_finish(acc, rs, out, take_sqrt);
}

// CG update x += alpha p, r -= alpha ap with alpha = s_an / s_ad from device
// memory, then *out = ||r|| (owned). Skips the update when |s_ad| < DBL_MIN
// (pcg.hpp:119-124 returns there) and writes *out = -1 so the host can tell.
__global__ void __launch_bounds__(kThreads) cg_update_kernel(VecDesc L, double* __restrict__ x,
                                                              double* __restrict__ r, const double* __restrict__ p,
                                                              const double* __restrict__ ap, const double* s_an,
                                                              const double* s_ad, RedScratch rs, double* out)
{
    const double ad = *s_ad;
    if (fabs(ad) < DBL_MIN) {
        if (blockIdx.x == 0 && threadIdx.x == 0) *out = -1.0;
        return;
    }
    const double  alpha  = *s_an / ad;
    double        acc    = 0.0;
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    for (int s = 0; s < L.nseg; ++s) {
        const VecSeg S = L.seg[s];
        for (int c = 0; c < S.ncomp; ++c) {
            const int64_t o = S.offset + c * S.stride;
            for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < S.n; i += stride) {
                x[o + i]        = x[o + i] + alpha * p[o + i];
                const double rv = r[o + i] - alpha * ap[o + i];
                r[o + i]        = rv;
                if (S.owned[lat_of(i, S.rdiv)]) acc += rv * rv;
            }
        }
    }
    block_finish(acc, rs, out, 1);
}

// p = z + (s_num / s_den) p
__global__ void p_update_kernel(int64_t n, double* __restrict__ p, const double* __restrict__ z, const double* s_num,
                                const double* s_den)
{
    const double  beta   = *s_num / *s_den;
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
        p[i] = z[i] + beta * p[i];
}

// v -= scale * (*s) on n entries
__global__ void sub_scalar_kernel(int64_t n, double* __restrict__ v, const double* s, double scale)
{
    const double  c      = scale * *s;
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) v[i] -= c;
}

template <typename T>
__global__ void scale_recip_kernel(int64_t n, T* __restrict__ y, const T* __restrict__ x, const double* s)
{
    const T       f      = static_cast<T>(1.0 / *s);
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) y[i] = f * x[i];
}

template <typename T, bool FIRST>
__global__ void cheb_kernel(int64_t n, T* __restrict__ x, T* __restrict__ d, const T* __restrict__ b,
                            const T* __restrict__ ax, const T* __restrict__ invd, T alpha, T beta)
{
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const T z  = (b[i] - ax[i]) * invd[i];
        const T dn = FIRST ? alpha * z : alpha * z + beta * d[i];
        d[i]       = dn;
        x[i]       = x[i] + dn;
    }
}

template <typename T>
__global__ void mul_kernel(int64_t n, T* __restrict__ y, const T* __restrict__ a, const T* __restrict__ b, T c)
{
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
        y[i] = c * (a[i] * b[i]);
}

__global__ void multi_axpy_kernel(int64_t n, double* __restrict__ x, AxpyList L)
{
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        double acc = 0.0;
        for (int k = 0; k < L.m; ++k) acc = acc + L.y[k] * L.z[k][i];
        x[i] = x[i] + acc;
    }
}

__device__ __forceinline__ uint64_t splitmix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

template <typename T>
struct CompPtrs {
    T* p[4];
};

template <typename T>
__global__ void random_kernel(int64_t n, int ncomp, CompPtrs<T> v, int nr, const int32_t* __restrict__ canon_lat,
                              uint64_t seed)
{
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    for (int c = 0; c < ncomp; ++c)
        for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
            const uint64_t lat = static_cast<uint64_t>(i / nr), r = static_cast<uint64_t>(i % nr);
            const uint64_t gid = (static_cast<uint64_t>(canon_lat[lat]) * nr + r) * ncomp + c;
            const uint64_t z   = splitmix64(seed + (gid + 1) * 0x9E3779B97F4A7C15ull);
            const double   u   = static_cast<double>(z >> 11) * (1.0 / 9007199254740992.0);
            v.p[c][i]          = static_cast<T>(2.0 * u - 1.0);
        }
}

template <typename T>
__global__ void nonfinite_kernel(int64_t n, const T* __restrict__ a, int* flag)
{
    bool          bad    = false;
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
        if (!isfinite(static_cast<double>(a[i]))) bad = true;
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicExch(flag, 1);
}

// f32 -> f64 with a non-finite flag (the FGMRES NaN/Inf check of the
// preconditioner output, fgmres.hpp:191-210, folded into the conversion).
__global__ void widen_check_kernel(int64_t n, const float* __restrict__ in, double* __restrict__ out, int* flag)
{
    bool          bad    = false;
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double v = static_cast<double>(in[i]);
        if (!isfinite(v)) bad = true;
        out[i] = v;
    }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicExch(flag, 1);
}

// ---------------------------------------------------------------------------
// Coarsest-grid CG in one cluster launch.
// ---------------------------------------------------------------------------
__host__ __device__ constexpr int woff_c(int w, int n, int k)
{
    constexpr int t[2][6][3] = {{{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {0, 1, 1}},
                                {{1, 1, 0}, {0, 1, 0}, {1, 0, 0}, {1, 1, 1}, {0, 1, 1}, {1, 0, 1}}};
    return t[w][n][k];
}

// Cluster-wide barrier; release / acquire at cluster scope orders the global
// memory accesses of all threads of the cluster around it.
__device__ __forceinline__ void cluster_barrier()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}
__device__ __forceinline__ unsigned cluster_rank()
{
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ unsigned cluster_ncta()
{
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
    return r;
}

constexpr int kPcgThreads = 1024;
constexpr int kPcgMaxCta  = 16;

// Sum of v over the cluster; every thread returns the same value (partials are
// summed in rank order).
__device__ double cluster_sum(double v, double* partials, int& buf, unsigned rank, unsigned ncta, double* red)
{
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int k = 0; k < kPcgThreads / 32; ++k) s += red[k];
        partials[buf * kPcgMaxCta + rank] = s;
    }
    cluster_barrier();
    double tot = 0.0;
    for (unsigned k = 0; k < ncta; ++k) tot += __ldcg(partials + buf * kPcgMaxCta + k);
    buf ^= 1;
    return tot;
}

// Per-CTA view of the coarsest level: this CTA's cells [c0, c0 + cnt), their
// node indices (int32, [w * 6 + n][local cell]) and their matrices (packed
// value-major, in shared memory when they fit, else the global array).
struct PcgView {
    int            c0, cnt, cpc;
    const int32_t* node;  // shared, [12][cpc]
    const double*  mb;    // matrices of local cell lc at mb[p * ms + lc]
    int64_t        ms;
};

__device__ __forceinline__ int pidx_rt(int a, int b)
{
    const int i = a < b ? a : b, j = a < b ? b : a;
    return i * (37 - i) / 2 + (j - i);
}

// dst (zero on entry) = A src with the interface sum; ends with a cluster barrier.
__device__ void pcg_matvec(const CoarsePcgArgs& A, const PcgView& V, const double* src, double* dst, unsigned g,
                           unsigned G)
{
    const int64_t S     = A.stride;
    const int     items = 36 * V.cnt;
    for (int it = threadIdx.x; it < items; it += blockDim.x) {
        const int lc   = it % V.cnt;
        const int rest = it / V.cnt;
        const int w    = rest & 1;
        const int a    = rest >> 1;
        double    acc  = 0.0;
#pragma unroll
        for (int b = 0; b < 18; ++b) {
            const int nb = b % 6, cb = b / 6;
            acc += V.mb[static_cast<int64_t>(w * 171 + pidx_rt(a, b)) * V.ms + lc] *
                   __ldcg(src + cb * S + V.node[(w * 6 + nb) * V.cpc + lc]);
        }
        const int na = a % 6, ca = a / 6;
        atomicAdd(dst + ca * S + V.node[(w * 6 + na) * V.cpc + lc], acc);
    }
    cluster_barrier();
    const int nr     = A.nr;
    const int iitems = A.num_classes * nr * 3;
    for (int it = static_cast<int>(g); it < iitems; it += static_cast<int>(G)) {
        const int r    = it % nr;
        const int rest = it / nr;
        const int c    = rest % 3;
        const int cls  = rest / 3;
        const int b0 = A.off[cls], b1 = A.off[cls + 1];
        double*   v  = dst + c * S;
        double    s  = 0.0;
        for (int m = b0; m < b1; ++m) s += __ldcg(v + static_cast<int64_t>(A.mem[m]) * nr + r);
        for (int m = b0; m < b1; ++m) v[static_cast<int64_t>(A.mem[m]) * nr + r] = s;
    }
    cluster_barrier();
}

__global__ void __launch_bounds__(kPcgThreads, 1) coarse_pcg_kernel(CoarsePcgArgs A)
{
    extern __shared__ __align__(16) unsigned char pcg_smem[];
    __shared__ double red[kPcgThreads / 32];
    const unsigned    rank = cluster_rank(), ncta = cluster_ncta();
    const unsigned    g = rank * kPcgThreads + threadIdx.x, G = ncta * kPcgThreads;
    const int         nl = A.nl, nr = A.nr;
    const int         nc = 10 * (nl - 1) * (nl - 1) * (nr - 1);

    PcgView V;
    V.cpc = A.cells_per_cta;
    V.c0  = static_cast<int>(rank) * V.cpc;
    V.cnt = nc - V.c0 < V.cpc ? nc - V.c0 : V.cpc;
    if (V.cnt < 0) V.cnt = 0;
    int32_t* node = reinterpret_cast<int32_t*>(pcg_smem);
    for (int i = threadIdx.x; i < 12 * V.cpc; i += blockDim.x) {
        const int lc = i % V.cpc, k = i / V.cpc;
        int32_t   v  = 0;
        if (lc < V.cnt) {
            const int cell = V.c0 + lc;
            const int r    = cell % (nr - 1);
            int       t    = cell / (nr - 1);
            const int y    = t % (nl - 1);
            t /= (nl - 1);
            const int x = t % (nl - 1), d = t / (nl - 1);
            const int w = k / 6, n = k % 6;
            v = static_cast<int32_t>(
                node_index(nl, nr, d, x + woff_c(w, n, 0), y + woff_c(w, n, 1), r + woff_c(w, n, 2)));
        }
        node[i] = v;
    }
    V.node = node;
    if (A.mats_in_smem) {
        double* ms = reinterpret_cast<double*>(pcg_smem + A.node_bytes);
        for (int i = threadIdx.x; i < 342 * V.cpc; i += blockDim.x) {
            const int lc = i % V.cpc, p = i / V.cpc;
            ms[i]        = lc < V.cnt ? A.mats[static_cast<int64_t>(p) * nc + V.c0 + lc] : 0.0;
        }
        V.mb = ms;
        V.ms = V.cpc;
    } else {
        V.mb = A.mats + V.c0;
        V.ms = nc;
    }
    __syncthreads();

    const int      n = static_cast<int>(A.n), n3 = 3 * n;
    const int64_t  S = A.stride;
    const uint32_t unr = static_cast<uint32_t>(nr);
    int            buf = 0;
    for (int i = static_cast<int>(g); i < n3; i += static_cast<int>(G)) {
        const int c = i / n, j = i - c * n;
        A.ap[c * S + j] = 0.0;
    }
    cluster_barrier();
    pcg_matvec(A, V, A.x, A.ap, g, G);
    double acc = 0.0;
    for (int i = static_cast<int>(g); i < n3; i += static_cast<int>(G)) {
        const int     c = i / n, j = i - c * n;
        const int64_t o = c * S + j;
        const double  rv = __ldcg(A.b + o) - __ldcg(A.ap + o);
        A.r[o]           = rv;
        A.p[o]           = rv;
        A.ap[o]          = 0.0;
        if (A.owned[static_cast<uint32_t>(j) / unr]) acc += rv * rv;
    }
    double       rr   = cluster_sum(acc, A.partials, buf, rank, ncta, red);
    const double init = sqrt(rr);
    double       res  = init;
    int          its  = 0;
    if (!(init < A.atol)) {
        double an = rr;
        for (int it = 1; it <= A.max_iter; ++it) {
            pcg_matvec(A, V, A.p, A.ap, g, G);
            acc = 0.0;
            for (int i = static_cast<int>(g); i < n3; i += static_cast<int>(G)) {
                const int     c = i / n, j = i - c * n;
                const int64_t o = c * S + j;
                if (A.owned[static_cast<uint32_t>(j) / unr]) acc += __ldcg(A.ap + o) * __ldcg(A.p + o);
            }
            const double ad = cluster_sum(acc, A.partials, buf, rank, ncta, red);
            if (fabs(ad) < DBL_MIN) break;
            const double alpha = an / ad;
            acc                = 0.0;
            for (int i = static_cast<int>(g); i < n3; i += static_cast<int>(G)) {
                const int     c = i / n, j = i - c * n;
                const int64_t o = c * S + j;
                A.x[o]          = __ldcg(A.x + o) + alpha * __ldcg(A.p + o);
                const double rv = __ldcg(A.r + o) - alpha * __ldcg(A.ap + o);
                A.r[o]          = rv;
                if (A.owned[static_cast<uint32_t>(j) / unr]) acc += rv * rv;
            }
            rr  = cluster_sum(acc, A.partials, buf, rank, ncta, red);
            res = sqrt(rr);
            its = it;
            if (res / init <= A.rtol || res < A.atol) break;
            const double bn = rr;
            if (fabs(an) < DBL_MIN) break;
            const double beta = bn / an;
            for (int i = static_cast<int>(g); i < n3; i += static_cast<int>(G)) {
                const int     c = i / n, j = i - c * n;
                const int64_t o = c * S + j;
                A.p[o]          = __ldcg(A.r + o) + beta * __ldcg(A.p + o);
                A.ap[o]         = 0.0;
            }
            cluster_barrier();
            an = bn;
        }
    }
    if (g == 0 && A.stats) {
        A.stats[0] = static_cast<double>(its);
        A.stats[1] = init;
        A.stats[2] = res;
    }
}

// ---------------------------------------------------------------------------
// Coarsest CG with the vectors replicated in every CTA's shared memory (levels
// with up to ~2000 nodes, e.g. level 2). Each CTA applies its cells' matrices
// to its local copy of p into a local partial (shared-memory atomics); the
// partials are summed slice by slice over distributed shared memory and the
// sums broadcast back, so after two cluster barriers every CTA holds the full
// A p. Dots and vector updates then run on local copies, identically (same
// data, same order) in every CTA, and need no further communication.
// ---------------------------------------------------------------------------
// Block-wide sum returned to every thread. The warp sums go to one of two
// buffers in turn, so a single barrier suffices: a buffer is written again
// only two calls later, after every thread has passed the barrier of the call
// in between (and so has finished reading it).
__device__ double block_sum_all(double v, double* red, int& parity)
{
    v           = warp_sum(v);
    double* buf = red + (parity & 1) * 32;
    ++parity;
    if ((threadIdx.x & 31) == 0) buf[threadIdx.x >> 5] = v;
    __syncthreads();
    // every warp folds the warp sums with the same butterfly, so all threads
    // (and all CTAs holding the same data) get identical bits
    const int lane = threadIdx.x & 31;
    return warp_sum(lane < static_cast<int>(blockDim.x >> 5) ? buf[lane] : 0.0);
}

// Owned-entry dot over the three components (own: one byte per entry of a
// component, 1 where the lateral node is owned).
__device__ __forceinline__ double owned_dot(const double* a, const double* b, int n, const uint8_t* own, double* red,
                                             int& parity)
{
    double acc = 0.0;
#pragma unroll
    for (int c = 0; c < 3; ++c)
        for (int j = threadIdx.x; j < n; j += blockDim.x)
            if (own[j]) acc += a[c * n + j] * b[c * n + j];
    return block_sum_all(acc, red, parity);
}

// Shared-memory tables of the replicated coarsest CG, built once per launch
// (the work assignment does not change between iterations).
struct RepTables {
    const int32_t* node;     // [12][cpc]: node index of wedge node (w, n) of local cell lc
    const uint8_t* own;      // [n]
    const int32_t* mv_code;  // [items]: lc | (w * 18 + a) << 16
    const int32_t* if_base;  // [iitems]: c * n + r of interface item
    const int32_t* if_cls;   // [iitems]
    const int32_t* cls_off;  // [num_classes + 1]
    const int32_t* mem_nr;   // [members]: member lateral index * nr
    int            items, iitems, cpc, c0;
};

// dst = A src (all CTAs end with the same full vector). part must be zero on
// entry and is zero again on return. xch: blockDim.x doubles of scratch.
// Each matvec item is one row a of one wedge's 18 x 18 matrix for one local
// cell, read from the row-major copy mats_full[(w * 18 + a) * 18 + b][cell].
__device__ void rep_matvec(const CoarsePcgArgs& A, const RepTables& R, const double* src, double* dst, double* part,
                           double* xch, int n, int n3, int nc, cg::cluster_group& cluster)
{
    for (int k = 0; k < 2; ++k) {
        const int it = threadIdx.x + k * blockDim.x;
        if (it >= R.items) break;
        const int      code = R.mv_code[it];
        const int      lc = code & 0xffff, wa = code >> 16;
        const int      w = wa >= 18 ? 1 : 0, a = wa - 18 * w;
        const double*  row  = A.mats_full + static_cast<int64_t>(wa) * 18 * nc + (R.c0 + lc);
        const int32_t* nd   = R.node + w * 6 * R.cpc + lc;
        int            idx[6];
#pragma unroll
        for (int nb = 0; nb < 6; ++nb) idx[nb] = nd[nb * R.cpc];
        double acc = 0.0;
#pragma unroll
        for (int b = 0; b < 18; ++b) acc += __ldg(row + static_cast<int64_t>(b) * nc) * src[(b / 6) * n + idx[b % 6]];
        atomicAdd(part + (a / 6) * n + idx[a % 6], acc);
    }
    cluster.sync();
    // This CTA sums slice [e0, e1) over all CTAs' partials: thread t reads
    // element e0 + t % sl from the CTAs k, k + ng, ... (k = t / sl), the ng
    // group sums are combined in a fixed order, and the same thread layout
    // writes the result to every CTA's dst.
    const unsigned ncta = cluster.num_blocks(), rank = cluster.block_rank();
    const int      sl   = (n3 + static_cast<int>(ncta) - 1) / static_cast<int>(ncta);
    const int      e0 = static_cast<int>(rank) * sl, e1 = e0 + sl < n3 ? e0 + sl : n3;
    const int      len = e1 > e0 ? e1 - e0 : 0;
    if (sl <= static_cast<int>(blockDim.x)) {
        int ng = static_cast<int>(blockDim.x) / sl;
        if (ng > static_cast<int>(ncta)) ng = static_cast<int>(ncta);
        const int t = threadIdx.x, k = t / sl, i = t - k * sl;
        if (k < ng) {
            double v = 0.0;
            if (i < len)
                for (int c = k; c < static_cast<int>(ncta); c += ng) v += cluster.map_shared_rank(part, c)[e0 + i];
            xch[t] = v;
        }
        __syncthreads();
        if (t < len) {  // column t: group sums in order k = 0, 1, ...
            double v = xch[t];
            for (int g = 1; g < ng; ++g) v += xch[g * sl + t];
            xch[t] = v;
        }
        __syncthreads();
        if (k < ng && i < len)
            for (int c = k; c < static_cast<int>(ncta); c += ng) cluster.map_shared_rank(dst, c)[e0 + i] = xch[i];
    } else {
        for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
            double v = 0.0;
            for (unsigned c = 0; c < ncta; ++c) v += cluster.map_shared_rank(part, c)[e];
            for (unsigned c = 0; c < ncta; ++c) cluster.map_shared_rank(dst, c)[e] = v;
        }
    }
    cluster.sync();
    for (int e = threadIdx.x; e < n3; e += blockDim.x) part[e] = 0.0;
    // interface sums: every copy of an interface node gets the class sum
    for (int it = threadIdx.x; it < R.iitems; it += blockDim.x) {
        double*   v  = dst + R.if_base[it];
        const int cl = R.if_cls[it];
        const int b0 = R.cls_off[cl], b1 = R.cls_off[cl + 1];
        double    s  = 0.0;
        for (int m = b0; m < b1; ++m) s += v[R.mem_nr[m]];
        for (int m = b0; m < b1; ++m) v[R.mem_nr[m]] = s;
    }
    __syncthreads();
}

__global__ void __launch_bounds__(kPcgThreads, 1) coarse_pcg_rep_kernel(CoarsePcgArgs A)
{
    extern __shared__ __align__(16) unsigned char pcg_smem[];
    __shared__ double   red[2 * 32];
    __shared__ double   xch[kPcgThreads];
    int                 parity  = 0;
    cg::cluster_group   cluster = cg::this_cluster();
    const unsigned      rank = cluster.block_rank(), ncta = cluster.num_blocks();
    const int           nl = A.nl, nr = A.nr;
    const int           nc = 10 * (nl - 1) * (nl - 1) * (nr - 1);
    const int           n = static_cast<int>(A.n), n3 = 3 * n;
    const int64_t       S = A.stride;
    const uint64_t      rdiv = reciprocal_nr(nr);

    // shared layout (offsets as in pcg_config): 4 vectors, node table, item
    // codes, interface tables, ownership bytes
    double*  p_s  = reinterpret_cast<double*>(pcg_smem);
    double*  r_s  = p_s + n3;
    double*  ap_s = r_s + n3;
    double*  pt_s = ap_s + n3;
    int32_t* node = reinterpret_cast<int32_t*>(pt_s + n3);
    const int cpc = A.cells_per_cta;
    int32_t*  mv_code = node + 12 * cpc;
    const int items   = 36 * cpc;
    const int iitems  = A.num_classes * nr * 3;
    int32_t*  if_base = mv_code + items;
    int32_t*  if_cls  = if_base + iitems;
    int32_t*  cls_off = if_cls + iitems;
    const int nmem    = A.num_classes > 0 ? A.off[A.num_classes] : 0;
    int32_t*  mem_nr  = cls_off + A.num_classes + 1;
    uint8_t*  own     = reinterpret_cast<uint8_t*>(mem_nr + nmem);

    RepTables R;
    R.cpc = cpc;
    R.c0  = static_cast<int>(rank) * cpc;
    int cnt = nc - R.c0 < cpc ? nc - R.c0 : cpc;
    if (cnt < 0) cnt = 0;
    R.items  = 36 * cnt;
    R.iitems = iitems;
    for (int i = threadIdx.x; i < 12 * cpc; i += blockDim.x) {
        const int lc = i % cpc, k = i / cpc;
        int32_t   v  = 0;
        if (lc < cnt) {
            const int cell = R.c0 + lc;
            const int r    = cell % (nr - 1);
            int       t    = cell / (nr - 1);
            const int y    = t % (nl - 1);
            t /= (nl - 1);
            const int x = t % (nl - 1), d = t / (nl - 1);
            const int w = k / 6, nn = k % 6;
            v = static_cast<int32_t>(
                node_index(nl, nr, d, x + woff_c(w, nn, 0), y + woff_c(w, nn, 1), r + woff_c(w, nn, 2)));
        }
        node[i] = v;
    }
    for (int it = threadIdx.x; it < R.items; it += blockDim.x) {
        const int lc = it % cnt, wa = it / cnt;  // wa = w * 18 + a
        mv_code[it]  = lc | (wa << 16);
    }
    for (int it = threadIdx.x; it < iitems; it += blockDim.x) {
        const int r = it % nr, rest = it / nr, c = rest % 3, cl = rest / 3;
        if_base[it] = c * n + r;
        if_cls[it]  = cl;
    }
    for (int i = threadIdx.x; i <= A.num_classes; i += blockDim.x) cls_off[i] = A.off[i];
    for (int m = threadIdx.x; m < nmem; m += blockDim.x) mem_nr[m] = A.mem[m] * nr;
    for (int j = threadIdx.x; j < n; j += blockDim.x) own[j] = A.owned[lat_of(j, rdiv)] ? 1 : 0;
    R.node    = node;
    R.own     = own;
    R.mv_code = mv_code;
    R.if_base = if_base;
    R.if_cls  = if_cls;
    R.cls_off = cls_off;
    R.mem_nr  = mem_nr;

    // slice of x this CTA updates: at most one entry per thread
    const int sl = (n3 + static_cast<int>(ncta) - 1) / static_cast<int>(ncta);
    const int x0 = static_cast<int>(rank) * sl, x1 = x0 + sl < n3 ? x0 + sl : n3;
    int       xe = -1;
    int64_t   xg = 0;
    if (x0 + static_cast<int>(threadIdx.x) < x1) {
        xe          = x0 + threadIdx.x;
        const int c = xe / n, j = xe - c * n;
        xg          = c * S + j;
    }

    // r = b - A x, p = r
#pragma unroll
    for (int c = 0; c < 3; ++c)
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            p_s[c * n + j]  = A.x[c * S + j];
            pt_s[c * n + j] = 0.0;
        }
    __syncthreads();
    rep_matvec(A, R, p_s, ap_s, pt_s, xch, n, n3, nc, cluster);
#pragma unroll
    for (int c = 0; c < 3; ++c)
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            const double rv = A.b[c * S + j] - ap_s[c * n + j];
            r_s[c * n + j]  = rv;
            p_s[c * n + j]  = rv;
        }
    __syncthreads();
    double       rr   = owned_dot(r_s, r_s, n, own, red, parity);
    const double init = sqrt(rr);
    double       res  = init;
    int          its  = 0;
    if (!(init < A.atol)) {
        double an = rr;
        for (int it = 1; it <= A.max_iter; ++it) {
            rep_matvec(A, R, p_s, ap_s, pt_s, xch, n, n3, nc, cluster);
            const double ad = owned_dot(ap_s, p_s, n, own, red, parity);
            if (fabs(ad) < DBL_MIN) break;
            const double alpha = an / ad;
            if (xe >= 0) A.x[xg] += alpha * p_s[xe];
            for (int e = threadIdx.x; e < n3; e += blockDim.x) r_s[e] = r_s[e] - alpha * ap_s[e];
            __syncthreads();
            rr  = owned_dot(r_s, r_s, n, own, red, parity);
            res = sqrt(rr);
            its = it;
            if (res / init <= A.rtol || res < A.atol) break;
            const double bn = rr;
            if (fabs(an) < DBL_MIN) break;
            const double beta = bn / an;
            for (int e = threadIdx.x; e < n3; e += blockDim.x) p_s[e] = r_s[e] + beta * p_s[e];
            __syncthreads();
            an = bn;
        }
    }
    if (rank == 0 && threadIdx.x == 0 && A.stats) {
        A.stats[0] = static_cast<double>(its);
        A.stats[1] = init;
        A.stats[2] = res;
    }
    // no CTA may leave while others still read its shared memory
    cluster.sync();
}

// Row-major copy of packed symmetric wedge matrices:
// full[(w * 18 + a) * 18 + b][cell] = packed[w * 171 + pidx(a, b)][cell].
__global__ void unpack_full_kernel(int nc, const double* __restrict__ packed, double* __restrict__ full)
{
    const int64_t total = static_cast<int64_t>(2) * 324 * nc;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int cell = static_cast<int>(i % nc);
        const int rab  = static_cast<int>(i / nc);
        const int w = rab / 324, ab = rab % 324, a = ab / 18, b = ab % 18;
        full[i]     = packed[static_cast<int64_t>(w * 171 + pidx_rt(a, b)) * nc + cell];
    }
}

__global__ void inject_kernel(int nlc, int nrc, const double* __restrict__ fine, double* __restrict__ coarse,
                              int reciprocal)
{
    const int     nlf = 2 * nlc - 1, nrf = 2 * nrc - 1;
    const int64_t n   = 10ll * nlc * nlc * nrc;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int r = static_cast<int>(i % nrc);
        int64_t   t = i / nrc;
        const int y = static_cast<int>(t % nlc);
        t /= nlc;
        const int    x = static_cast<int>(t % nlc);
        const int    d = static_cast<int>(t / nlc);
        const double v = fine[node_index(nlf, nrf, d, 2 * x, 2 * y, 2 * r)];
        coarse[i]      = reciprocal ? 1.0 / v : v;
    }
}

__global__ void cell_average_kernel(int nlc, int nrc, const double* __restrict__ fine, double* __restrict__ coarse)
{
    const int     nlf = 2 * nlc - 1, nrf = 2 * nrc - 1;
    const int64_t n   = 10ll * (nlc - 1) * (nlc - 1) * (nrc - 1);
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int r = static_cast<int>(i % (nrc - 1));
        int64_t   t = i / (nrc - 1);
        const int y = static_cast<int>(t % (nlc - 1));
        t /= (nlc - 1);
        const int x = static_cast<int>(t % (nlc - 1));
        const int d = static_cast<int>(t / (nlc - 1));
        double    s = 0.0;
        for (int c = 0; c < 8; ++c)
            s += fine[node_index(nlf - 1, nrf - 1, d, 2 * x + (c & 1), 2 * y + ((c >> 1) & 1), 2 * r + (c >> 2))];
        coarse[i] = 0.125 * s;
    }
}

// Strong boundary treatment of a velocity right-hand side: Dirichlet rows
// zeroed, free-slip normal components removed (n = unit lateral coordinate).
__global__ void enforce_bcs_kernel(int nl, int nr, const double* __restrict__ coords, int bc_cmb, int bc_surf,
                                   CompPtrs<double> v)
{
    const int lat = blockIdx.x * blockDim.x + threadIdx.x;
    if (lat >= 10 * nl * nl) return;
    const double* c = coords + static_cast<int64_t>(lat) * 3;
    const double  m = sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
    const double  n[3] = {c[0] / m, c[1] / m, c[2] / m};
    for (int side = 0; side < 2; ++side) {
        const int     bc = side == 0 ? bc_cmb : bc_surf;
        const int64_t id = static_cast<int64_t>(lat) * nr + (side == 0 ? 0 : nr - 1);
        if (bc == 1) {
            for (int k = 0; k < 3; ++k) v.p[k][id] = 0.0;
        } else if (bc == 2) {
            const double dn = n[0] * v.p[0][id] + n[1] * v.p[1][id] + n[2] * v.p[2][id];
            for (int k = 0; k < 3; ++k) v.p[k][id] -= dn * n[k];
        }
    }
}

inline int grid_for(int64_t n)
{
    int64_t b = (n + kThreads - 1) / kThreads;
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

int solver_partials_size() { return kBlocks; }

template <typename T>
int vec_dot(const VecDesc& L, const T* a, const T* b, double* out_dev, RedScratch rs, bool take_sqrt, cudaStream_t st)
{
    vdot_kernel<T><<<kBlocks, kThreads, 0, st>>>(L, a, b, rs, out_dev, take_sqrt ? 1 : 0);
    return launch_status();
}
template int vec_dot<double>(const VecDesc&, const double*, const double*, double*, RedScratch, bool, cudaStream_t);
template int vec_dot<float>(const VecDesc&, const float*, const float*, double*, RedScratch, bool, cudaStream_t);

int mgs_step(const VecDesc& L, double* w, const double* v_sub, const double* h_sub, const double* v_dot, double* out,
             RedScratch rs, cudaStream_t st)
{
    if (v_sub && v_dot)
        mgs_kernel<true, true><<<kBlocks, kThreads, 0, st>>>(L, w, v_sub, h_sub, v_dot, rs, out, 0);
    else if (v_dot)
        mgs_kernel<false, true><<<kBlocks, kThreads, 0, st>>>(L, w, v_sub, h_sub, v_dot, rs, out, 0);
    else if (v_sub)
        mgs_kernel<true, false><<<kBlocks, kThreads, 0, st>>>(L, w, v_sub, h_sub, v_dot, rs, out, 1);
    else
        mgs_kernel<false, false><<<kBlocks, kThreads, 0, st>>>(L, w, v_sub, h_sub, v_dot, rs, out, 1);
    return launch_status();
}

int cg_update(const VecDesc& L, double* x, double* r, const double* p, const double* ap, const double* s_an,
              const double* s_ad, double* out, RedScratch rs, cudaStream_t st)
{
    cg_update_kernel<<<kBlocks, kThreads, 0, st>>>(L, x, r, p, ap, s_an, s_ad, rs, out);
    return launch_status();
}

int sub_scalar(int64_t n, double* v, const double* s_dev, double scale, cudaStream_t st)
{
    sub_scalar_kernel<<<grid_for(n), kThreads, 0, st>>>(n, v, s_dev, scale);
    return launch_status();
}

int p_update(int64_t n, double* p, const double* z, const double* s_num, const double* s_den, cudaStream_t st)
{
    p_update_kernel<<<grid_for(n), kThreads, 0, st>>>(n, p, z, s_num, s_den);
    return launch_status();
}

template <typename T>
int scale_by_recip(int64_t n, T* y, const T* x, const double* s_dev, cudaStream_t st)
{
    scale_recip_kernel<T><<<grid_for(n), kThreads, 0, st>>>(n, y, x, s_dev);
    return launch_status();
}
template int scale_by_recip<double>(int64_t, double*, const double*, const double*, cudaStream_t);
template int scale_by_recip<float>(int64_t, float*, const float*, const double*, cudaStream_t);

template <typename T>
int cheb_step(int64_t n, T* x, T* d, const T* b, const T* ax, const T* invdiag, T alpha, T beta, bool first,
              cudaStream_t st)
{
    if (first)
        cheb_kernel<T, true><<<grid_for(n), kThreads, 0, st>>>(n, x, d, b, ax, invdiag, alpha, beta);
    else
        cheb_kernel<T, false><<<grid_for(n), kThreads, 0, st>>>(n, x, d, b, ax, invdiag, alpha, beta);
    return launch_status();
}
template int cheb_step<double>(int64_t, double*, double*, const double*, const double*, const double*, double, double,
                               bool, cudaStream_t);
template int cheb_step<float>(int64_t, float*, float*, const float*, const float*, const float*, float, float, bool,
                              cudaStream_t);

template <typename T>
int vec_mul(int64_t n, T* y, const T* a, const T* b, T c, cudaStream_t st)
{
    mul_kernel<T><<<grid_for(n), kThreads, 0, st>>>(n, y, a, b, c);
    return launch_status();
}
template int vec_mul<double>(int64_t, double*, const double*, const double*, double, cudaStream_t);
template int vec_mul<float>(int64_t, float*, const float*, const float*, float, cudaStream_t);

int multi_axpy(int64_t n, double* x, const AxpyList& list, cudaStream_t st)
{
    if (list.m < 0 || list.m > kMaxAxpy) return -1;
    if (list.m == 0) return 0;
    multi_axpy_kernel<<<grid_for(n), kThreads, 0, st>>>(n, x, list);
    return launch_status();
}

template <typename T>
int random_fill(int64_t n, int ncomp, T* const* comps, int nr, const int32_t* canon_lat, uint64_t seed,
                cudaStream_t st)
{
    if (ncomp < 1 || ncomp > 4) return -1;
    CompPtrs<T> v{};
    for (int c = 0; c < ncomp; ++c) v.p[c] = comps[c];
    random_kernel<T><<<grid_for(n), kThreads, 0, st>>>(n, ncomp, v, nr, canon_lat, seed);
    return launch_status();
}
template int random_fill<double>(int64_t, int, double* const*, int, const int32_t*, uint64_t, cudaStream_t);
template int random_fill<float>(int64_t, int, float* const*, int, const int32_t*, uint64_t, cudaStream_t);

template <typename T>
int flag_nonfinite(int64_t n, const T* a, int* flag_dev, cudaStream_t st)
{
    nonfinite_kernel<T><<<grid_for(n), kThreads, 0, st>>>(n, a, flag_dev);
    return launch_status();
}
template int flag_nonfinite<double>(int64_t, const double*, int*, cudaStream_t);
template int flag_nonfinite<float>(int64_t, const float*, int*, cudaStream_t);

int widen_check(int64_t n, const float* in, double* out, int* flag_dev, cudaStream_t st)
{
    widen_check_kernel<<<grid_for(n), kThreads, 0, st>>>(n, in, out, flag_dev);
    return launch_status();
}

namespace {
using PcgKernel = void (*)(CoarsePcgArgs);

// cluster size (16 when the device allows non-portable clusters of this
// kernel with the given shared memory, else 8)
int pcg_cluster_size(PcgKernel kernel, size_t smem)
{
    int size = 8;
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess) {
        cudaLaunchConfig_t  cfg = {};
        cudaLaunchAttribute at[1];
        at[0].id               = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = kPcgMaxCta;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.gridDim            = dim3(kPcgMaxCta);
        cfg.blockDim           = dim3(kPcgThreads);
        cfg.dynamicSmemBytes   = smem;
        cfg.attrs              = at;
        cfg.numAttrs           = 1;
        int nclusters          = 0;
        if (cudaOccupancyMaxActiveClusters(&nclusters, kernel, &cfg) == cudaSuccess && nclusters > 0)
            size = kPcgMaxCta;
    }
    cudaGetLastError();
    return size;
}

struct PcgConfig {
    int       cs = 0, cpc = 0, in_smem = 0;
    size_t    node_bytes = 0, smem = 0;
    PcgKernel kernel = nullptr;
};

// Launch configuration for a coarsest level (nodes per component n, nc
// cells), decided once per level size (function attributes and occupancy
// queries stay out of launches, so the launch can be captured in a graph).
// Levels whose four vectors fit in shared memory run the replicated kernel.
int pcg_config(int n, int nc, int nr, int ncls, int nmem, PcgConfig& out)
{
    static std::mutex                                           mu;
    // per device: the function attributes set below belong to the current device
    static std::map<std::tuple<int, int, int, int, int, int>, PcgConfig> cache;
    std::lock_guard<std::mutex>                                      lock(mu);
    int                                                              dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return -2;
    const auto key = std::make_tuple(dev, n, nc, nr, ncls, nmem);
    auto                                                        it  = cache.find(key);
    if (it != cache.end()) {
        out = it->second;
        return 0;
    }
    constexpr size_t kSmemLimit = 200 * 1024;
    PcgConfig        c;
    const size_t     vec_bytes = static_cast<size_t>(4) * 3 * n * sizeof(double);
    auto             layout    = [&](int cs) {
        c.cs         = cs;
        c.cpc        = (nc + cs - 1) / cs;
        c.node_bytes = (static_cast<size_t>(48) * c.cpc + 15) / 16 * 16;
        // replicated kernel tables: item codes, interface items (base, class),
        // class offsets, member indices, ownership bytes
        const size_t iitems = static_cast<size_t>(ncls) * nr * 3;
        const size_t tables = sizeof(int32_t) * (36 * static_cast<size_t>(c.cpc) + 2 * iitems + ncls + 1 + nmem) + n;
        const size_t rep    = vec_bytes + c.node_bytes + (tables + 15) / 16 * 16;
        if (rep <= kSmemLimit && 36 * c.cpc <= 2 * kPcgThreads) {
            c.kernel  = coarse_pcg_rep_kernel;
            c.smem    = rep;
            c.in_smem = 0;
        } else {
            c.kernel  = coarse_pcg_kernel;
            c.smem    = c.node_bytes + static_cast<size_t>(342 * 8) * c.cpc;
            c.in_smem = c.smem <= kSmemLimit ? 1 : 0;
            if (!c.in_smem) c.smem = c.node_bytes;
        }
    };
    layout(kPcgMaxCta);
    for (PcgKernel k : {static_cast<PcgKernel>(coarse_pcg_kernel), static_cast<PcgKernel>(coarse_pcg_rep_kernel)})
        if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kSmemLimit)) !=
            cudaSuccess) {
            cudaGetLastError();
            return -2;
        }
    if (pcg_cluster_size(c.kernel, c.smem) != kPcgMaxCta) layout(8);
    if (c.node_bytes > kSmemLimit) return -1;
    cache[key] = c;
    out        = c;
    return 0;
}
}  // namespace

int coarse_pcg_prepare(int nl, int nr, int num_classes, int num_members)
{
    PcgConfig c;
    return pcg_config(10 * nl * nl * nr, 10 * (nl - 1) * (nl - 1) * (nr - 1), nr, num_classes, num_members, c);
}

int coarse_pcg_uses_full_matrices(int nl, int nr, int num_classes, int num_members)
{
    PcgConfig c;
    if (pcg_config(10 * nl * nl * nr, 10 * (nl - 1) * (nl - 1) * (nr - 1), nr, num_classes, num_members, c) != 0)
        return 0;
    return c.kernel == coarse_pcg_rep_kernel ? 1 : 0;
}

int coarse_matrices_unpack(int nc, const double* packed, double* full, cudaStream_t st)
{
    unpack_full_kernel<<<1184, 256, 0, st>>>(nc, packed, full);
    return launch_status();
}

int coarse_pcg(const CoarsePcgArgs& args_in, cudaStream_t st)
{
    CoarsePcgArgs args = args_in;
    const int     nc   = 10 * (args.nl - 1) * (args.nl - 1) * (args.nr - 1);
    PcgConfig     c;
    const int     rc = pcg_config(static_cast<int>(args.n), nc, args.nr, args.num_classes, args.num_members, c);
    if (rc != 0) return rc;
    if (c.kernel == coarse_pcg_rep_kernel && args.mats_full == nullptr) return -1;
    args.cells_per_cta = c.cpc;
    args.node_bytes    = static_cast<int>(c.node_bytes);
    args.mats_in_smem  = c.in_smem;
    cudaLaunchConfig_t  cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id               = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = c.cs;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.gridDim            = dim3(c.cs);
    cfg.blockDim           = dim3(kPcgThreads);
    cfg.dynamicSmemBytes   = c.smem;
    cfg.stream             = st;
    cfg.attrs              = at;
    cfg.numAttrs           = 1;
    note_launch();
    if (cudaLaunchKernelEx(&cfg, c.kernel, args) != cudaSuccess) {
        cudaGetLastError();
        return -2;
    }
    return 0;
}

int coarse_pcg_partials_size() { return 2 * kPcgMaxCta; }

int enforce_velocity_bcs(int nl, int nr, const double* coords, int bc_cmb, int bc_surf, double* const* v,
                         cudaStream_t st)
{
    CompPtrs<double> p{};
    for (int k = 0; k < 3; ++k) p.p[k] = v[k];
    const int n = 10 * nl * nl;
    enforce_bcs_kernel<<<(n + 127) / 128, 128, 0, st>>>(nl, nr, coords, bc_cmb, bc_surf, p);
    return launch_status();
}

int coefficient_inject(int nlc, int nrc, const double* fine, double* coarse, bool reciprocal, cudaStream_t st)
{
    inject_kernel<<<grid_for(10ll * nlc * nlc * nrc), kThreads, 0, st>>>(nlc, nrc, fine, coarse, reciprocal ? 1 : 0);
    return launch_status();
}

int cell_coefficient_average(int nlc, int nrc, const double* fine, double* coarse, cudaStream_t st)
{
    cell_average_kernel<<<grid_for(10ll * nlc * nlc * nrc), kThreads, 0, st>>>(nlc, nrc, fine, coarse);
    return launch_status();
}

}  // namespace tn
