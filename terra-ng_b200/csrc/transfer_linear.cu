// Linear multigrid transfers between level l (fine) and l-1 (coarse) on the thick shell (sm_100a).
//
// Semantics of the reference's ProlongationLinear / RestrictionLinear (fe/wedge/operators/shell/
// prolongation_linear.hpp, restriction_linear.hpp) with the weights of prolongation_linear_weights
// (fe/wedge/shell/grid_transfer_linear.hpp:13-157), which interpolate affine functions exactly on the curved
// shell:
//   * a fine node on a coarse node copies it;
//   * a fine node radially between two coarse nodes of its own column takes (1 - nu, nu) with
//     nu = (|x_f| - |x_bot|) / (|x_top| - |x_bot|);
//   * any other fine node lies on a facet spanned by two coarse columns (the vertical, horizontal or
//     anti-diagonal edge of the diamond's triangulation) and takes 0.5 (1 - nu) from each bottom node and
//     0.5 nu from each top node, nu measured against the chord midpoints 0.5 (x_0 + x_1) of the two columns;
//   * the radial bracket is r_bot = r_f / 2, except on the outer shell (r_bot = r_f / 2 - 1), where the weights
//     extrapolate and can be negative.
// The weights depend only on the fine node, so they are computed once per level (FP64, from the fine level's
// coordinates) into a table of two values per fine node.
//
// The vector transfers apply the scalar transfer to every component. (The reference's ProlongationVecLinear
// leaves its component loop after the first component on coarse-aligned and radially aligned nodes, an early
// return inside the loop, so its second and third components miss those contributions; ProlongationLinear per
// component is the consistent operator and the one its scalar multigrid tests use.)
//
//   prolongate_linear_add: fine += P coarse, one thread per fine node gathering 1, 2 or 4 coarse values; the
//                          lateral pair is summed first so every interface copy rounds identically.
//   restrict_linear_owned: coarse = P^T (owned fine), one thread per coarse node gathering from the fine
//                          nodes whose prolongation reads it (7 lateral x 5 radial candidates), non-owned fine
//                          duplicates masked, no atomics; the caller completes it with the interface sum.
#include "tn_device.cuh"
#include "tn_kernels.hpp"
#include "tn_wedge_math.cuh"

namespace tn {
namespace {

constexpr int kMaxComp = 4;
constexpr int kThreads = 256;

template <typename T>
struct LPtr {
    const T* in[kMaxComp];
    T*       out[kMaxComp];
};

// Coarse parents of fine node (x, y, r): lateral pair (x0, y0), (x1, y1) (equal when aligned) and radial
// bracket; kind 0: on a coarse node, 1: radially aligned, 2: on a facet.
struct Parents {
    int kind, x0, y0, x1, y1, rb, rt;
};
__host__ __device__ __forceinline__ Parents parents(int x, int y, int r, int nrf)
{
    Parents p;
    if ((x & 1) == 0 && (y & 1) == 0 && (r & 1) == 0) {
        p.kind = 0;
        p.x0 = p.x1 = x / 2;
        p.y0 = p.y1 = y / 2;
        p.rb = p.rt = r / 2;
        return p;
    }
    p.rb = r < nrf - 1 ? r / 2 : r / 2 - 1;
    p.rt = p.rb + 1;
    if ((x & 1) == 0 && (y & 1) == 0) {
        p.kind = 1;
        p.x0 = p.x1 = x / 2;
        p.y0 = p.y1 = y / 2;
    } else if ((x & 1) == 0) {  // vertical edge
        p.kind = 2;
        p.x0 = x / 2, p.x1 = x / 2, p.y0 = y / 2, p.y1 = y / 2 + 1;
    } else if ((y & 1) == 0) {  // horizontal edge
        p.kind = 2;
        p.x0 = x / 2, p.x1 = x / 2 + 1, p.y0 = y / 2, p.y1 = y / 2;
    } else {  // anti-diagonal edge
        p.kind = 2;
        p.x0 = x / 2 + 1, p.x1 = x / 2, p.y0 = y / 2, p.y1 = y / 2 + 1;
    }
    return p;
}

__device__ __forceinline__ double norm3(double a, double b, double c) { return sqrt(a * a + b * b + c * c); }

__global__ void __launch_bounds__(kThreads) weights_kernel(int nlf, int nrf, const double* __restrict__ coords,
                                                           const double* __restrict__ radii, int n, Decoder rad,
                                                           Decoder lat, double* __restrict__ w)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int d, x, y, r, col;
    decode4(i, rad, lat, d, x, y, r, col);
    const Parents p = parents(x, y, r, nrf);
    double        w0 = 1.0, w1 = 0.0;
    if (p.kind != 0) {
        const double* uf = coords + 3 * node_index(nlf, 1, d, x, y, 0);
        const double  rf = radii[r];
        const double  nf = norm3(uf[0] * rf, uf[1] * rf, uf[2] * rf);
        const double  rbot = radii[2 * p.rb], rtop = radii[2 * p.rt];
        double        nb, nt;
        if (p.kind == 1) {
            nb = norm3(uf[0] * rbot, uf[1] * rbot, uf[2] * rbot);
            nt = norm3(uf[0] * rtop, uf[1] * rtop, uf[2] * rtop);
        } else {
            const double* u0 = coords + 3 * node_index(nlf, 1, d, 2 * p.x0, 2 * p.y0, 0);
            const double* u1 = coords + 3 * node_index(nlf, 1, d, 2 * p.x1, 2 * p.y1, 0);
            double        cb[3], ct[3];
            for (int k = 0; k < 3; ++k) {
                cb[k] = 0.5 * (u0[k] * rbot + u1[k] * rbot);
                ct[k] = 0.5 * (u0[k] * rtop + u1[k] * rtop);
            }
            nb = norm3(cb[0], cb[1], cb[2]);
            nt = norm3(ct[0], ct[1], ct[2]);
        }
        const double nu = (nf - nb) / (nt - nb);
        w0              = p.kind == 1 ? 1.0 - nu : 0.5 * (1.0 - nu);
        w1              = p.kind == 1 ? nu : 0.5 * nu;
    }
    w[2 * static_cast<int64_t>(i)]     = w0;
    w[2 * static_cast<int64_t>(i) + 1] = w1;
}

template <typename T>
__global__ void __launch_bounds__(kThreads) prolongate_linear_kernel(int nlf, int nrf, int ncomp, LPtr<T> P,
                                                                     const T* __restrict__ w, int n, Decoder rad,
                                                                     Decoder lat)
{
    const int nlc = (nlf + 1) / 2, nrc = (nrf + 1) / 2;
    const int i   = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int d, x, y, r, col;
    decode4(i, rad, lat, d, x, y, r, col);
    const Parents p  = parents(x, y, r, nrf);
    const T       w0 = w[2 * static_cast<int64_t>(i)], w1 = w[2 * static_cast<int64_t>(i) + 1];
    for (int c = 0; c < ncomp; ++c) {
        const T* src = P.in[c];
        T        v;
        if (p.kind == 0) {
            v = src[node_index(nlc, nrc, d, p.x0, p.y0, p.rb)];
        } else if (p.kind == 1) {
            v = w0 * src[node_index(nlc, nrc, d, p.x0, p.y0, p.rb)] + w1 * src[node_index(nlc, nrc, d, p.x0, p.y0, p.rt)];
        } else {
            const T bot = src[node_index(nlc, nrc, d, p.x0, p.y0, p.rb)] + src[node_index(nlc, nrc, d, p.x1, p.y1, p.rb)];
            const T top = src[node_index(nlc, nrc, d, p.x0, p.y0, p.rt)] + src[node_index(nlc, nrc, d, p.x1, p.y1, p.rt)];
            v           = w0 * bot + w1 * top;
        }
        P.out[c][i] += v;
    }
}

template <typename T>
__global__ void __launch_bounds__(kThreads) restrict_linear_kernel(int nlf, int nrf, int ncomp,
                                                                   const uint8_t* __restrict__ owned, LPtr<T> P,
                                                                   const T* __restrict__ w, int n, Decoder rad,
                                                                   Decoder lat)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int d, xc, yc, rc, col;
    decode4(i, rad, lat, d, xc, yc, rc, col);
    constexpr int ox[7] = {0, -1, -1, 0, 1, 1, 0};
    constexpr int oy[7] = {0, 0, 1, 1, 0, -1, -1};
    T             acc[kMaxComp];
    for (int c = 0; c < ncomp; ++c) acc[c] = T(0);
    for (int o = 0; o < 7; ++o) {
        const int xf = 2 * xc + ox[o], yf = 2 * yc + oy[o];
        if (xf < 0 || xf >= nlf || yf < 0 || yf >= nlf) continue;
        if (!owned[lat_index3(nlf, d, xf, yf)]) continue;
        for (int rf = 2 * rc - 2; rf <= 2 * rc + 2; ++rf) {
            if (rf < 0 || rf >= nrf) continue;
            const Parents p = parents(xf, yf, rf, nrf);
            const bool    lat_hit = (p.x0 == xc && p.y0 == yc) || (p.x1 == xc && p.y1 == yc);
            if (!lat_hit) continue;
            const int64_t fi = node_index(nlf, nrf, d, xf, yf, rf);
            T             wgt;
            if (p.kind == 0) {
                if (p.rb != rc) continue;
                wgt = T(1);
            } else if (p.rb == rc) {
                wgt = w[2 * fi];
            } else if (p.rt == rc) {
                wgt = w[2 * fi + 1];
            } else {
                continue;
            }
            for (int c = 0; c < ncomp; ++c) acc[c] += wgt * P.in[c][fi];
        }
    }
    for (int c = 0; c < ncomp; ++c) P.out[c][i] = acc[c];
}

inline int launch_status(int kernels = 1)
{
    note_launch(kernels);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

}  // namespace

int linear_transfer_weights(int nlf, int nrf, const double* coords_fine, const double* radii_fine, double* w,
                            cudaStream_t st)
{
    const int n = 10 * nlf * nlf * nrf;
    weights_kernel<<<(n + kThreads - 1) / kThreads, kThreads, 0, st>>>(nlf, nrf, coords_fine, radii_fine, n,
                                                                       Decoder(nrf), Decoder(nlf), w);
    return launch_status();
}

template <typename T>
int prolongate_linear_add(int nlf, int nrf, int ncomp, const T* w, const T* const* coarse, T* const* fine,
                          cudaStream_t st)
{
    if (ncomp < 1 || ncomp > kMaxComp) return -1;
    LPtr<T> P{};
    for (int c = 0; c < ncomp; ++c) {
        P.in[c]  = coarse[c];
        P.out[c] = fine[c];
    }
    const int n = 10 * nlf * nlf * nrf;
    prolongate_linear_kernel<T><<<(n + kThreads - 1) / kThreads, kThreads, 0, st>>>(nlf, nrf, ncomp, P, w, n,
                                                                                    Decoder(nrf), Decoder(nlf));
    return launch_status();
}

template <typename T>
int restrict_linear_owned(int nlf, int nrf, int ncomp, const uint8_t* owned_lat_fine, const T* w,
                          const T* const* fine, T* const* coarse, cudaStream_t st)
{
    if (ncomp < 1 || ncomp > kMaxComp) return -1;
    LPtr<T> P{};
    for (int c = 0; c < ncomp; ++c) {
        P.in[c]  = fine[c];
        P.out[c] = coarse[c];
    }
    const int nlc = (nlf + 1) / 2, nrc = (nrf + 1) / 2;
    const int n   = 10 * nlc * nlc * nrc;
    restrict_linear_kernel<T><<<(n + kThreads - 1) / kThreads, kThreads, 0, st>>>(
        nlf, nrf, ncomp, owned_lat_fine, P, w, n, Decoder(nrc), Decoder(nlc));
    return launch_status();
}

template int prolongate_linear_add<double>(int, int, int, const double*, const double* const*, double* const*,
                                           cudaStream_t);
template int prolongate_linear_add<float>(int, int, int, const float*, const float* const*, float* const*,
                                          cudaStream_t);
template int restrict_linear_owned<double>(int, int, int, const uint8_t*, const double*, const double* const*,
                                           double* const*, cudaStream_t);
template int restrict_linear_owned<float>(int, int, int, const uint8_t*, const float*, const float* const*,
                                          float* const*, cudaStream_t);

}  // namespace tn
