// P1-iso-P2 / P1 coupling blocks and mass matrices (FP64 and FP32).
//
//   divergence B   : fine velocity (level L) -> coarse pressure (level L-1)
//                    p_i += -|det J| shape_coarse_i div u   (divergence_kerngen.hpp:519-778)
//   gradient   B^T : coarse pressure -> fine velocity
//                    u_{n,d} += -|det J| g_{n,d} p_interp   (gradient_kerngen.hpp:498-759)
//   lumped k-mass  : diag of the 6-point k-weighted pressure mass (kmass.hpp:98-181)
//   vector mass    : 6-point mass matrix applied per component (vector_mass.hpp:60-150)
//
// B and B^T run in two passes through one scalar per fine wedge (described
// before the kernels below) on flat grids, with the factorised wedge Jacobian
// of the epsilon-div-div kernel from per-level geometry tables. The mass
// matrices run one thread per fine cell and add with native FP64/FP32 global
// atomics (set-up only). The coarse node of fine wedge node i is
// (x/2, y/2, r/2) + the fine wedge's node offset, with the reference's
// shape_coarse(i, r%2, fine_lateral_wedge_idx(x, y, w)) weights; this keeps
// B and B^T exact transposes of each other and of the reference.
#include <algorithm>

#include "tn_device.cuh"
#include "tn_kernels.hpp"
#include "tn_wedge_math.cuh"

namespace tn {
namespace {

__host__ __device__ constexpr int woff(int w, int n, int k)
{
    // WEDGE_NODE_OFF (kernel_helpers.hpp:291-312)
    constexpr int t[2][6][3] = {{{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {0, 1, 1}},
                                {{1, 1, 0}, {0, 1, 0}, {1, 0, 0}, {1, 1, 1}, {0, 1, 1}, {1, 0, 1}}};
    return t[w][n][k];
}

// fine_lateral_wedge_idx (kernel_helpers.hpp:600-608)
__host__ __device__ __forceinline__ int fine_lat_wedge(int x, int y, int w)
{
    constexpr int idx[2][2][2] = {{{0, 1}, {2, 3}}, {{3, 2}, {1, 0}}};
    return idx[w][y & 1][x & 1];
}

// shape_coarse(i, frw, flw, centroid) (integrands.hpp:250-393) at (1/3, 1/3, 0).
template <typename T>
__host__ __device__ __forceinline__ T shape_coarse_centroid(int i, int frw, int flw)
{
    const T xi = T(1) / T(3), eta = T(1) / T(3);
    T       lat;
    switch (i % 3) {
    case 0:
        lat = flw == 0 ? T(-0.5) * eta - T(0.5) * xi + T(1) : (flw == 3 ? T(0.5) * eta + T(0.5) * xi : T(-0.5) * eta - T(0.5) * xi + T(0.5));
        break;
    case 1: lat = flw == 1 ? T(0.5) * xi + T(0.5) : (flw == 3 ? T(0.5) - T(0.5) * xi : T(0.5) * xi); break;
    default: lat = flw == 2 ? T(0.5) * eta + T(0.5) : (flw == 3 ? T(0.5) - T(0.5) * eta : T(0.5) * eta); break;
    }
    T rad;
    if (i / 3 == 0)
        rad = frw == 0 ? T(0.75) : T(0.25);
    else
        rad = frw == 0 ? T(0.25) : T(0.75);
    return lat * rad;
}

template <typename T>
struct CouplingArgs {
    int      nl, nr;  // fine level
    const T* coords;  // fine unit-sphere coords
    const T* colgeo;  // fine per-column wedge geometry (20 values per column)
    const T* radgeo;  // fine per-radial-cell alpha, 1/(6 hdr), r_mid^2 hdr
    const T* radii;   // fine radii
    int      bc_cmb, bc_surf;
    const T* u[3];    // fine velocity (divergence input / gradient output)
    T*       uo[3];
    const T* p;       // coarse pressure (gradient input)
    T*       po;      // coarse pressure (divergence output)
};

template <typename T>
__device__ __forceinline__ void unit_normal(const T* coords, int nl, int d, int x, int y, T (&n)[3])
{
    const T* c = coords + lat_index3(nl, d, x, y) * 3;
    n[0]       = c[0];
    n[1]       = c[1];
    n[2]       = c[2];
}

// Both blocks go through one scalar per fine wedge, stored in a scratch array
// wedge_val[2 * fine_cell + w]:
//   B  : -|det J_w| div_w(u), div_w = tr(G) = e1.a + e2.b + e3.D (the
//        factorised velocity gradient of the epsilon-div-div kernel);
//   B^T: -|det J_w| p_interp,w with p_interp the coarse-pressure interpolation
//        at the fine wedge's centroid.
// Pass 1 runs one thread per fine cell; pass 2 distributes: B adds the 16
// fine wedges of a coarse cell into its 8 corners (8 atomics per coarse cell),
// B^T gathers, per fine node, the up to 12 wedges around it (no atomics,
// every node written once). Every kernel runs one CTA per lateral column
// (grid = (y, x, diamond)) with threads along r, so the lateral geometry is
// one broadcast per CTA and the radial factors come from the level's table.

// Flat grids of 256 threads, one thread per fine cell / coarse cell / fine
// node in storage order (r fastest), so warps read consecutive radial
// entries and no thread idles; indices are decoded with Decoder (exact
// reciprocal multiplications).
constexpr int kCouplingThreads = 256;

template <typename T>
struct Pair;
template <>
struct Pair<double> {
    using type = double2;
};
template <>
struct Pair<float> {
    using type = float2;
};

// B, pass 1: one thread per fine cell. All 24 corner values are loaded
// before any arithmetic (the kernel is bound by load latency, so every load
// of a cell is in flight at once); the lateral geometry is read from L1 where
// it is used rather than held in registers.
template <typename T>
__global__ void __launch_bounds__(kCouplingThreads) div_cells_kernel(CouplingArgs<T> A, T* __restrict__ wv, int nc,
                                                                        Decoder rad, Decoder lat)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nc) return;
    const int nl = A.nl, nr = A.nr;
    int       d, x, y, r, col;
    decode4(i, rad, lat, d, x, y, r, col);
    const T* G = A.colgeo + static_cast<int64_t>(col) * 20;
    T        u[4][2][3];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        // node offsets fit in 32 bits (10 nl^2 nr < 2^31 up to level 8)
        const int id = static_cast<int>(node_index(nl, nr, d, x + (q & 1), y + (q >> 1), r));
#pragma unroll
        for (int s2 = 0; s2 < 2; ++s2)
#pragma unroll
            for (int c = 0; c < 3; ++c) u[q][s2][c] = A.u[c][id + s2];
    }
    const bool at_cmb = r == 0, at_surf = r + 1 == nr - 1;
    const int  bcf    = at_cmb ? A.bc_cmb : (at_surf ? A.bc_surf : 0);
    if (bcf == 1 || bcf == 2) {
        const int bside = at_cmb ? 0 : 1;
        // compile-time side index (a runtime index would move u to local memory)
#pragma unroll
        for (int sd = 0; sd < 2; ++sd) {
            if (sd != bside) continue;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                if (bcf == 1) {
                    u[q][sd][0] = u[q][sd][1] = u[q][sd][2] = T(0);
                } else {
                    T nn[3];
                    unit_normal<T>(A.coords, nl, d, x + (q & 1), y + (q >> 1), nn);
                    const T un = u[q][sd][0] * nn[0] + u[q][sd][1] * nn[1] + u[q][sd][2] * nn[2];
#pragma unroll
                    for (int c = 0; c < 3; ++c) u[q][sd][c] -= un * nn[c];
                }
            }
        }
    }
    const T alpha = A.radgeo[3 * r], beta = A.radgeo[3 * r + 1], dfac = A.radgeo[3 * r + 2];
    T       out[2];
#pragma unroll
    for (int w = 0; w < 2; ++w) {
        const T*  g  = G + 10 * w;
        const int q0 = wedge_corner(w, 0), q1 = wedge_corner(w, 1), q2 = wedge_corner(w, 2);
        T         div = T(0);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const T S0 = u[q0][0][c] + u[q0][1][c], S1 = u[q1][0][c] + u[q1][1][c], S2 = u[q2][0][c] + u[q2][1][c];
            const T Dc = (u[q0][1][c] - u[q0][0][c]) + (u[q1][1][c] - u[q1][0][c]) + (u[q2][1][c] - u[q2][0][c]);
            div += alpha * (__ldg(g + c) * (S1 - S0) + __ldg(g + 3 + c) * (S2 - S0)) + beta * __ldg(g + 6 + c) * Dc;
        }
        out[w] = -(__ldg(g + 9) * dfac) * div;
    }
    using V = typename Pair<T>::type;
    V o;
    o.x                         = out[0];
    o.y                         = out[1];
    reinterpret_cast<V*>(wv)[i] = o;
}

// B, pass 2: one thread per coarse cell adds its 16 fine wedges into its 8
// corners.
template <typename T>
__global__ void __launch_bounds__(kCouplingThreads) div_scatter_kernel(CouplingArgs<T> A, const T* __restrict__ wv,
                                                                       int ncc, Decoder rad, Decoder lat)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ncc) return;
    const int nl = A.nl, nr = A.nr, nlc = (nl + 1) / 2, nrc = (nr + 1) / 2;
    int       d, X, Y, R, col;
    decode4(i, rad, lat, d, X, Y, R, col);
    using V = typename Pair<T>::type;
    T acc[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) acc[k] = T(0);
#pragma unroll
    for (int f = 0; f < 8; ++f) {
        const int     x = 2 * X + (f & 1), y = 2 * Y + ((f >> 1) & 1), c = f >> 2, r = 2 * R + c;
        const int64_t fc = node_index(nl - 1, nr - 1, d, x, y, r);
        const V       pv = reinterpret_cast<const V*>(wv)[fc];
#pragma unroll
        for (int w = 0; w < 2; ++w) {
            const T   pre = w == 0 ? pv.x : pv.y;
            const int flw = fine_lat_wedge(x, y, w);
#pragma unroll
            for (int j = 0; j < 6; ++j)
                acc[woff(w, j, 0) + 2 * woff(w, j, 1) + 4 * woff(w, j, 2)] += pre * shape_coarse_centroid<T>(j, c, flw);
        }
    }
#pragma unroll
    for (int k = 0; k < 8; ++k)
        atomicAdd(&A.po[node_index(nlc, nrc, d, X + (k & 1), Y + ((k >> 1) & 1), R + (k >> 2))], acc[k]);
}

// B^T, pass 1: one thread per fine cell, p interpolated at both wedge centroids.
template <typename T>
__global__ void __launch_bounds__(kCouplingThreads) grad_cells_kernel(CouplingArgs<T> A, T* __restrict__ wv, int nc,
                                                                      Decoder rad, Decoder lat)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nc) return;
    const int nl = A.nl, nr = A.nr, nlc = (nl + 1) / 2, nrc = (nr + 1) / 2;
    int       d, x, y, r, col;
    decode4(i, rad, lat, d, x, y, r, col);
    const T*  G    = A.colgeo + static_cast<int64_t>(col) * 20;
    const T   dfac = A.radgeo[3 * r + 2];
    const int X = x / 2, Y = y / 2, R = r / 2, frw = r & 1;
    T         pc[8];  // coarse cell corner pressures
#pragma unroll
    for (int k = 0; k < 8; ++k) pc[k] = A.p[node_index(nlc, nrc, d, X + (k & 1), Y + ((k >> 1) & 1), R + (k >> 2))];
    T out[2];
#pragma unroll
    for (int w = 0; w < 2; ++w) {
        const int flw = fine_lat_wedge(x, y, w);
        T         pi  = T(0);
#pragma unroll
        for (int j = 0; j < 6; ++j)
            pi += shape_coarse_centroid<T>(j, frw, flw) * pc[woff(w, j, 0) + 2 * woff(w, j, 1) + 4 * woff(w, j, 2)];
        out[w] = -(__ldg(G + 10 * w + 9) * dfac) * pi;
    }
    using V = typename Pair<T>::type;
    V o;
    o.x                            = out[0];
    o.y                            = out[1];
    reinterpret_cast<V*>(wv)[i] = o;
}

// B^T, pass 2: one thread per fine node gathers the up to 12 wedges around it.
template <typename T>
__global__ void __launch_bounds__(kCouplingThreads) grad_gather_kernel(CouplingArgs<T> A, const T* __restrict__ wv,
                                                                       int add, int nn, Decoder rad, Decoder lat)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nn) return;
    const int nl = A.nl, nr = A.nr;
    int       d, x, y, r, lcol;
    decode4(i, rad, lat, d, x, y, r, lcol);
    const bool on_cmb = r == 0, on_surf = r == nr - 1;
    const int  bcn    = on_cmb ? A.bc_cmb : (on_surf ? A.bc_surf : 0);
    T          o[3]   = {T(0), T(0), T(0)};
    if (bcn != 1) {
        // cell r above the node (node = its bottom, sign -1), cell r - 1 below (top, +1)
        const bool up = r <= nr - 2, dn = r >= 1;
        const T    al_up = up ? A.radgeo[3 * r] : T(0), sb_up = up ? -A.radgeo[3 * r + 1] : T(0);
        const T    al_dn = dn ? A.radgeo[3 * (r - 1)] : T(0), sb_dn = dn ? A.radgeo[3 * (r - 1) + 1] : T(0);
#pragma unroll
        for (int ab = 0; ab < 4; ++ab) {
            const int a = ab & 1, b = ab >> 1;
            const int xc = x - a, yc = y - b;
            if (xc < 0 || yc < 0 || xc > nl - 2 || yc > nl - 2) continue;
            const int col = (d * (nl - 1) + xc) * (nl - 1) + yc;
            const int q   = a + 2 * b;  // hex corner of the node in the cell
            const T*  G   = A.colgeo + static_cast<int64_t>(col) * 20;
            const int fc  = col * (nr - 1) + r;  // cell above; fc - 1 below
#pragma unroll
            for (int w = 0; w < 2; ++w) {
                const int m = w == 0 ? q : 3 - q;  // lateral index of corner q in wedge w
                if (m > 2) continue;
                const T* g    = G + 10 * w;
                const T  p_up = up ? wv[2 * fc + w] : T(0);
                const T  p_dn = dn ? wv[2 * fc - 2 + w] : T(0);
                const T  ca   = p_up * al_up + p_dn * al_dn;  // multiplies L_m
                const T  cb   = p_up * sb_up + p_dn * sb_dn;  // multiplies e3
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const T L = m == 0 ? -(__ldg(g + k) + __ldg(g + 3 + k)) : (m == 1 ? __ldg(g + k) : __ldg(g + 3 + k));
                    o[k] += ca * L + cb * __ldg(g + 6 + k);
                }
            }
        }
        if (bcn == 2) {
            T nv[3];
            unit_normal<T>(A.coords, nl, d, x, y, nv);
            const T on = o[0] * nv[0] + o[1] * nv[1] + o[2] * nv[2];
#pragma unroll
            for (int k = 0; k < 3; ++k) o[k] -= on * nv[k];
        }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) A.uo[k][i] = add ? A.uo[k][i] + o[k] : o[k];
}

// Radial factor table (one thread per radial cell).
template <typename T>
__global__ void radgeo_kernel(int nr, const T* radii, T* out)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nr - 1) return;
    const T r0 = radii[r], r1 = radii[r + 1];
    const T rm = T(0.5) * (r0 + r1), hdr = T(0.5) * (r1 - r0);
    out[3 * r]     = T(0.5) / rm;
    out[3 * r + 1] = T(1) / (T(6) * hdr);
    out[3 * r + 2] = rm * rm * hdr;
}

// Per-column wedge geometry table (column_geometry, 20 values per column).
template <typename T>
__global__ void colgeo_kernel(int nl, const T* coords, T* out)
{
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= 10 * (nl - 1) * (nl - 1)) return;
    const int y = col % (nl - 1);
    const int x = (col / (nl - 1)) % (nl - 1);
    const int d = col / ((nl - 1) * (nl - 1));
    column_geometry<T>(coords, nl, d, x, y, out + static_cast<int64_t>(col) * 20);
}

// Felippa 3x2 rule (quadrature.hpp:57-100).
__host__ __device__ constexpr double qp6(int q, int k)
{
    constexpr double t[6][3] = {{0.6666666666666666, 0.1666666666666667, -0.5773502691896257},
                                {0.1666666666666667, 0.6666666666666666, -0.5773502691896257},
                                {0.1666666666666667, 0.1666666666666667, -0.5773502691896257},
                                {0.6666666666666666, 0.1666666666666667, 0.5773502691896257},
                                {0.1666666666666667, 0.6666666666666666, 0.5773502691896257},
                                {0.1666666666666667, 0.1666666666666667, 0.5773502691896257}};
    return t[q][k];
}

// 6x6 wedge mass matrix with optional nodal coefficient (kmass.hpp:120-160,
// vector_mass.hpp:96-130), FP64 accumulation.
template <typename T>
__device__ void wedge_mass(const T* coords, int nl, int d, int x, int y, const T* radii, int r, int w, const T* kloc,
                           double (&M)[6][6])
{
    double p[3][3];
#pragma unroll
    for (int m = 0; m < 3; ++m) {
        const int q = wedge_corner(w, m);
        const T*  c = coords + lat_index3(nl, d, x + (q & 1), y + (q >> 1)) * 3;
        for (int i = 0; i < 3; ++i) p[m][i] = static_cast<double>(c[i]);
    }
    const double r1 = radii[r], r2 = radii[r + 1], grad_r = 0.5 * (r2 - r1);
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) M[i][j] = 0.0;
    for (int q = 0; q < 6; ++q) {
        const double xi = qp6(q, 0), eta = qp6(q, 1), zeta = qp6(q, 2);
        double       J[3][3];
        for (int i = 0; i < 3; ++i) {
            J[i][0] = p[1][i] - p[0][i];
            J[i][1] = p[2][i] - p[0][i];
            J[i][2] = (1 - xi - eta) * p[0][i] + xi * p[1][i] + eta * p[2][i];
        }
        double dl = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) - J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                    J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
        dl              = dl < 0 ? -dl : dl;
        const double rq = r1 + 0.5 * (r2 - r1) * (1 + zeta);
        double       N[6];
        const double lat[3] = {1.0 - xi - eta, xi, eta};
        for (int n = 0; n < 6; ++n) N[n] = lat[n % 3] * (n < 3 ? 0.5 * (1 - zeta) : 0.5 * (1 + zeta));
        double kev = 1.0;
        if (kloc) {
            kev = 0.0;
            for (int n = 0; n < 6; ++n) kev += N[n] * static_cast<double>(kloc[n]);
        }
        for (int i = 0; i < 6; ++i)
            for (int j = 0; j < 6; ++j) M[i][j] += 0.1666666666666667 * kev * (N[i] * N[j] * rq * rq * grad_r * dl);
    }
}

template <typename T>
__global__ void kmass_lumped_kernel(int nl, int nr, const T* coords, const T* radii, const T* k, T* diag)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y % (nl - 1), x = blockIdx.y / (nl - 1), d = blockIdx.z;
    if (r >= nr - 1) return;
    for (int w = 0; w < 2; ++w) {
        T kl[6];
        for (int n = 0; n < 6; ++n) kl[n] = k[node_index(nl, nr, d, x + woff(w, n, 0), y + woff(w, n, 1), r + woff(w, n, 2))];
        double M[6][6];
        wedge_mass<T>(coords, nl, d, x, y, radii, r, w, kl, M);
        for (int i = 0; i < 6; ++i) {
            double rs = 0;
            for (int j = 0; j < 6; ++j) rs += M[i][j];
            atomicAdd(&diag[node_index(nl, nr, d, x + woff(w, i, 0), y + woff(w, i, 1), r + woff(w, i, 2))],
                      static_cast<T>(rs));
        }
    }
}

template <typename T>
__global__ void vector_mass_kernel(int nl, int nr, const T* coords, const T* radii, CouplingArgs<T> A)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y % (nl - 1), x = blockIdx.y / (nl - 1), d = blockIdx.z;
    if (r >= nr - 1) return;
    for (int w = 0; w < 2; ++w) {
        double M[6][6];
        wedge_mass<T>(coords, nl, d, x, y, radii, r, w, nullptr, M);
        int64_t id[6];
        for (int n = 0; n < 6; ++n) id[n] = node_index(nl, nr, d, x + woff(w, n, 0), y + woff(w, n, 1), r + woff(w, n, 2));
        for (int c = 0; c < 3; ++c)
            for (int i = 0; i < 6; ++i) {
                double acc = 0;
                for (int j = 0; j < 6; ++j) acc += M[i][j] * static_cast<double>(A.u[c][id[j]]);
                atomicAdd(&A.uo[c][id[i]], static_cast<T>(acc));
            }
    }
}

inline int launch_status(int kernels = 1)
{
    note_launch(kernels);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

inline dim3 cell_grid(int nl, int nr, int threads) { return dim3((nr - 1 + threads - 1) / threads, (nl - 1) * (nl - 1), 10); }

}  // namespace

template <typename T>
static CouplingArgs<T> coupling_args(const CouplingLaunch<T>& p)
{
    CouplingArgs<T> a{};
    a.nl      = p.nl;
    a.nr      = p.nr;
    a.coords  = p.coords;
    a.colgeo  = p.colgeo;
    a.radgeo  = p.radgeo;
    a.radii   = p.radii;
    a.bc_cmb  = p.bc_cmb;
    a.bc_surf = p.bc_surf;
    for (int c = 0; c < 3; ++c) {
        a.u[c]  = p.u[c];
        a.uo[c] = p.u_out[c];
    }
    a.p  = p.p_in;
    a.po = p.p_out;
    return a;
}

template <typename T>
int divergence_apply(const CouplingLaunch<T>& p, cudaStream_t st)
{
    if (!p.wedge_scratch) return -1;
    if (!p.radgeo) return -1;
    const CouplingArgs<T> a   = coupling_args(p);
    const int             nlc = (p.nl + 1) / 2, nrc = (p.nr + 1) / 2;
    const int             nc  = 10 * (p.nl - 1) * (p.nl - 1) * (p.nr - 1);
    const int             ncc = 10 * (nlc - 1) * (nlc - 1) * (nrc - 1);
    constexpr int         B   = kCouplingThreads;
    div_cells_kernel<T><<<(nc + B - 1) / B, B, 0, st>>>(a, p.wedge_scratch, nc, Decoder(p.nr - 1), Decoder(p.nl - 1));
    div_scatter_kernel<T><<<(ncc + B - 1) / B, B, 0, st>>>(a, p.wedge_scratch, ncc, Decoder(nrc - 1),
                                                           Decoder(nlc - 1));
    return launch_status(2);
}

template <typename T>
int gradient_apply(const CouplingLaunch<T>& p, cudaStream_t st)
{
    if (!p.wedge_scratch) return -1;
    if (!p.radgeo) return -1;
    const CouplingArgs<T> a  = coupling_args(p);
    const int             nc = 10 * (p.nl - 1) * (p.nl - 1) * (p.nr - 1);
    const int             nn = 10 * p.nl * p.nl * p.nr;
    constexpr int         B  = kCouplingThreads;
    grad_cells_kernel<T><<<(nc + B - 1) / B, B, 0, st>>>(a, p.wedge_scratch, nc, Decoder(p.nr - 1), Decoder(p.nl - 1));
    grad_gather_kernel<T><<<(nn + B - 1) / B, B, 0, st>>>(a, p.wedge_scratch, p.add, nn, Decoder(p.nr),
                                                          Decoder(p.nl));
    return launch_status(2);
}

template <typename T>
int radial_geometry_table(int nr, const T* radii, T* out, cudaStream_t st)
{
    radgeo_kernel<T><<<(nr - 1 + 127) / 128, 128, 0, st>>>(nr, radii, out);
    return launch_status();
}
template int radial_geometry_table<double>(int, const double*, double*, cudaStream_t);
template int radial_geometry_table<float>(int, const float*, float*, cudaStream_t);

template <typename T>
int column_geometry_table(int nl, const T* coords, T* out, cudaStream_t st)
{
    const int n = 10 * (nl - 1) * (nl - 1);
    colgeo_kernel<T><<<(n + 127) / 128, 128, 0, st>>>(nl, coords, out);
    return launch_status();
}

template <typename T>
int kmass_lumped_add(int nl, int nr, const T* coords, const T* radii, const T* k, T* diag, cudaStream_t st)
{
    const int thr = nr - 1 >= 64 ? 64 : 32;
    kmass_lumped_kernel<T><<<cell_grid(nl, nr, thr), thr, 0, st>>>(nl, nr, coords, radii, k, diag);
    return launch_status();
}

template <typename T>
int vector_mass_add(int nl, int nr, const T* coords, const T* radii, const T* const* src, T* const* dst, cudaStream_t st)
{
    CouplingArgs<T> a{};
    for (int c = 0; c < 3; ++c) {
        a.u[c]  = src[c];
        a.uo[c] = dst[c];
    }
    const int thr = nr - 1 >= 64 ? 64 : 32;
    vector_mass_kernel<T><<<cell_grid(nl, nr, thr), thr, 0, st>>>(nl, nr, coords, radii, a);
    return launch_status();
}

#define TN_INST(T)                                                                                                 \
    template int divergence_apply<T>(const CouplingLaunch<T>&, cudaStream_t);                                     \
    template int gradient_apply<T>(const CouplingLaunch<T>&, cudaStream_t);                                       \
    template int column_geometry_table<T>(int, const T*, T*, cudaStream_t);                                       \
    template int kmass_lumped_add<T>(int, int, const T*, const T*, const T*, T*, cudaStream_t);                  \
    template int vector_mass_add<T>(int, int, const T*, const T*, const T* const*, T* const*, cudaStream_t);
TN_INST(double)
TN_INST(float)
#undef TN_INST

}  // namespace tn
