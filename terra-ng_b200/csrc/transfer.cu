// Constant-weight multigrid transfers between level l (fine) and l-1 (coarse).
//
// Weights are prolongation_constant_weight (fe/wedge/shell/
// grid_transfer_constant.hpp:24-89): linear interpolation on the anti-diagonal
// triangulation of each diamond, tensor product with linear interpolation in r.
//   prolongate_add : fine += P coarse   (ProlongationVecConstant, Add mode,
//                    prolongation_constant.hpp:146-191), here as a gather: one
//                    thread per fine node reading its 1..8 coarse parents, no atomics.
//   restrict_owned : coarse = P^T (owned fine)  (RestrictionVecConstant,
//                    restriction_constant.hpp:190-249): one thread per coarse
//                    node over its 21-point fine stencil, non-owned fine
//                    duplicates masked; the caller completes it with the coarse
//                    interface sum.
#include "tn_device.cuh"
#include "tn_kernels.hpp"
#include "tn_wedge_math.cuh"

namespace tn {
namespace {

constexpr int kMaxComp = 4;
template <typename T>
struct PtrSet {
    const T* in[kMaxComp];
    T*       out[kMaxComp];
};

// Flat grids: one thread per fine node (prolongation) or coarse node
// (restriction) in storage order, 256 threads per CTA, indices decoded with
// Decoder, so no thread of a radial column idles.
constexpr int kTransferThreads = 256;

template <typename T>
__global__ void __launch_bounds__(kTransferThreads) prolongate_kernel(int nlf, int nrf, int ncomp, PtrSet<T> P, int n,
                                                                      Decoder rad, Decoder lat)
{
    const int nlc = (nlf + 1) / 2, nrc = (nrf + 1) / 2;
    const int i   = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int d, x, y, r, col;
    decode4(i, rad, lat, d, x, y, r, col);
    // lateral parents (at most two) with weights
    int xa[2], ya[2], nlat;
    if ((x & 1) == 0 && (y & 1) == 0) {
        xa[0] = x / 2;
        ya[0] = y / 2;
        nlat  = 1;
    } else if ((y & 1) == 0) {
        xa[0] = (x - 1) / 2, ya[0] = y / 2;
        xa[1] = (x + 1) / 2, ya[1] = y / 2;
        nlat  = 2;
    } else if ((x & 1) == 0) {
        xa[0] = x / 2, ya[0] = (y - 1) / 2;
        xa[1] = x / 2, ya[1] = (y + 1) / 2;
        nlat  = 2;
    } else {
        xa[0] = (x + 1) / 2, ya[0] = (y - 1) / 2;
        xa[1] = (x - 1) / 2, ya[1] = (y + 1) / 2;
        nlat  = 2;
    }
    int       ra[2], nrad;
    const T   wl = nlat == 1 ? T(1) : T(0.5);
    if ((r & 1) == 0) {
        ra[0] = r / 2;
        nrad  = 1;
    } else {
        ra[0] = (r - 1) / 2;
        ra[1] = (r + 1) / 2;
        nrad  = 2;
    }
    const T       wr = nrad == 1 ? T(1) : T(0.5);
    const int64_t fi = i;
    // Copies of a diamond-edge node in different diamonds list their two
    // lateral parents in different orders. Summing the lateral pair first
    // (a two-term sum is the same in either order) and then the radial pair
    // (same order everywhere) gives every copy identical bits, so prolonged
    // vectors stay consistent on interface duplicates in FP32 as in FP64.
    for (int c = 0; c < ncomp; ++c) {
        T acc = T(0);
        for (int b = 0; b < nrad; ++b) {
            T lat = P.in[c][node_index(nlc, nrc, d, xa[0], ya[0], ra[b])];
            if (nlat == 2) lat += P.in[c][node_index(nlc, nrc, d, xa[1], ya[1], ra[b])];
            acc += lat;
        }
        P.out[c][fi] += wl * wr * acc;
    }
}

template <typename T>
__global__ void __launch_bounds__(kTransferThreads) restrict_kernel(int nlf, int nrf, int ncomp,
                                                                    const uint8_t* __restrict__ owned, PtrSet<T> P,
                                                                    int n, Decoder rad, Decoder lat)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int d, xc, yc, rc, col;
    decode4(i, rad, lat, d, xc, yc, rc, col);
    // 7-point lateral stencil (prolongation_constant_fine_grid_stencil_offsets_at_coarse_vertex)
    constexpr int ox[7] = {-1, -1, 0, 1, 1, 0, 0};
    constexpr int oy[7] = {0, 1, 1, 0, -1, -1, 0};
    T             acc[kMaxComp];
    for (int c = 0; c < ncomp; ++c) acc[c] = T(0);
#pragma unroll
    for (int o = 0; o < 7; ++o) {
        const int xf = 2 * xc + ox[o], yf = 2 * yc + oy[o];
        if (xf < 0 || xf >= nlf || yf < 0 || yf >= nlf) continue;
        if (!owned[lat_index3(nlf, d, xf, yf)]) continue;
        const T wl = (o == 6) ? T(1) : T(0.5);
#pragma unroll
        for (int dr = -1; dr <= 1; ++dr) {
            const int rf = 2 * rc + dr;
            if (rf < 0 || rf >= nrf) continue;
            const T       wgt = dr == 0 ? wl : T(0.5) * wl;
            const int64_t fi  = node_index(nlf, nrf, d, xf, yf, rf);
            for (int c = 0; c < ncomp; ++c) acc[c] += wgt * P.in[c][fi];
        }
    }
    const int64_t ci = i;
    for (int c = 0; c < ncomp; ++c) P.out[c][ci] = acc[c];
}

inline int launch_status(int kernels = 1)
{
    note_launch(kernels);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

}  // namespace

template <typename T>
int prolongate_add(int nlf, int nrf, int ncomp, const T* const* coarse, T* const* fine, cudaStream_t st)
{
    if (ncomp < 1 || ncomp > kMaxComp) return -1;
    PtrSet<T> P{};
    for (int c = 0; c < ncomp; ++c) {
        P.in[c]  = coarse[c];
        P.out[c] = fine[c];
    }
    const int n = 10 * nlf * nlf * nrf;
    prolongate_kernel<T><<<(n + kTransferThreads - 1) / kTransferThreads, kTransferThreads, 0, st>>>(
        nlf, nrf, ncomp, P, n, Decoder(nrf), Decoder(nlf));
    return launch_status();
}

template <typename T>
int restrict_owned(int nlf, int nrf, int ncomp, const uint8_t* owned_lat_fine, const T* const* fine, T* const* coarse,
                   cudaStream_t st)
{
    if (ncomp < 1 || ncomp > kMaxComp) return -1;
    PtrSet<T> P{};
    for (int c = 0; c < ncomp; ++c) {
        P.in[c]  = fine[c];
        P.out[c] = coarse[c];
    }
    const int nlc = (nlf + 1) / 2, nrc = (nrf + 1) / 2;
    const int n = 10 * nlc * nlc * nrc;
    restrict_kernel<T><<<(n + kTransferThreads - 1) / kTransferThreads, kTransferThreads, 0, st>>>(
        nlf, nrf, ncomp, owned_lat_fine, P, n, Decoder(nrc), Decoder(nlc));
    return launch_status();
}

template int prolongate_add<double>(int, int, int, const double* const*, double* const*, cudaStream_t);
template int prolongate_add<float>(int, int, int, const float* const*, float* const*, cudaStream_t);
template int restrict_owned<double>(int, int, int, const uint8_t*, const double* const*, double* const*, cudaStream_t);
template int restrict_owned<float>(int, int, int, const uint8_t*, const float* const*, float* const*, cudaStream_t);

}  // namespace tn
