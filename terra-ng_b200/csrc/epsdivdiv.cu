// epsilon-div-div wedge operator apply for sm_100a (FP64 and FP32).
//
// Semantics follow the reference's EpsilonDivDivKerngen (src/terra/fe/wedge/
// operators/shell/epsilon_divdiv_kerngen.hpp): 1-point centroid quadrature,
// k_eval = mean of the six nodal coefficients (or a per-cell Q0 value),
// Dirichlet rows reduced to their diagonal (:1569-1602), free-slip as
// P A P + diag_nn(A) n n^T on boundary nodes (:1638-2198), and a diagonal mode
// that applies diag(A) (rotated diagonal on free-slip nodes, :2008-2102).
//
// Formulation. The wedge Jacobian factorises as J = M diag(r_mid, r_mid, dr/2)
// with M = [p1-p0, p2-p0, (p0+p1+p2)/3] built from unit-sphere corners only
// (kernel_helpers.hpp:179-258). With M^{-T} = [e1 e2 e3] the physical gradient
// of node (m, side s) is g = alpha L_m + s beta e3, alpha = 1/(2 r_mid),
// beta = 1/(3 dr), L_1 = e1, L_2 = e2, L_0 = -(e1 + e2). The velocity gradient
// of a wedge is then G = e1 (x) a + e2 (x) b + e3 (x) D (alpha, beta folded in),
// the stress sigma = k|det J| (2 sym G - 2/3 tr G I), and the nodal outputs
// sigma g. About 110 flops per wedge instead of two 3x3 inversions plus the
// per-node gather/scatter of the reference.
//
// Work decomposition (one CTA = a tile of TY node lines in y x a chunk of CX
// node rows in x x all radial nodes of one diamond):
//   * lanes run along r (CPL consecutive radial cells per lane): coalesced
//     access to the r-fastest layout, radial node sums by warp shuffles;
//   * warp w owns cell strip y = y0 - 1 + w; strip-to-strip sums go through
//     shared memory, the strip left of the tile is recomputed (halo);
//   * the CTA sweeps x; the two cell columns that meet at a node row are
//     consecutive steps, so x sums are carried in registers;
//   * each new node row (TY + 2 columns x nr values, contiguous in global
//     memory) is staged by one TMA bulk copy per field into a 3-deep ring,
//     two rows ahead of use. Every node value is written once by its owner:
//     no atomics, no zeroing pass.
// Diamond-edge duplicates hold this diamond's partial sums afterwards; the
// interface-sum kernel completes them.
#include "tn_device.cuh"
#include "tn_kernels.hpp"
#include "tn_wedge_math.cuh"

#include <algorithm>
#include <atomic>
#include <mutex>
#include <type_traits>

namespace tn {
namespace {

// Warps per CTA (tile_y + 1): FP64 needs up to 255 registers per thread (8
// warps fill the register file), FP32 fits 12 warps.
// devices a process can drive (per-device launch caches)
constexpr int kMaxDevices = 64;

template <typename T>
struct MaxWarps;
template <>
struct MaxWarps<double> {
    static constexpr int value = 8;
};
template <>
struct MaxWarps<float> {
    static constexpr int value = 12;
};

// ---------------------------------------------------------------------------
// FP32 interior cells two at a time. A lane's radial cells c and c + 32 share
// their lateral geometry, so the arithmetic of hex_interior runs on float2
// pairs with the packed FP32 instructions of sm_100 (FFMA2 / FADD2 / FMUL2):
// one instruction per two cells. Subtraction is fma(b, -1, a), which rounds
// like a - b. The nodal outputs are assembled per corner: corners 0 and 3
// belong to one wedge each, corners 1 and 2 to both, with the lateral part
// lat and radial part rad giving bottom = lat - rad and top = lat + rad.
// ---------------------------------------------------------------------------
using f2 = float2;
__device__ __forceinline__ f2 p_add(f2 a, f2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ f2 p_sub(f2 a, f2 b) { return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a); }
__device__ __forceinline__ f2 p_mul(f2 a, f2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ f2 p_fma(f2 a, f2 b, f2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ f2 p_bc(float a) { return make_float2(a, a); }

__device__ __forceinline__ void hex_interior_x2(const f2 (&u)[4][2][3], const f2 (&ks)[4], f2 kcell, bool q0,
                                                const float* geo, f2 alpha, f2 beta, f2 dfac, f2 (&out)[4][2][3])
{
    f2 S[4][3], Dq[4][3];
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            S[q][c]  = p_add(u[q][0][c], u[q][1][c]);
            Dq[q][c] = p_sub(u[q][1][c], u[q][0][c]);
        }
    f2 v1w[2][3], v2w[2][3], wvw[2][3];
#pragma unroll
    for (int w = 0; w < 2; ++w) {
        const float* gw  = geo + 10 * w;
        const int    q0i = wedge_corner(w, 0), q1i = wedge_corner(w, 1), q2i = wedge_corner(w, 2);
        const f2     kv  = q0 ? kcell : p_add(p_add(ks[q0i], ks[q1i]), ks[q2i]);
        const f2     kw  = p_mul(kv, p_mul(dfac, p_bc(gw[9])));
        f2           E1[3], E2[3], E3[3], a[3], b[3], D[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            E1[i] = p_mul(alpha, p_bc(gw[i]));
            E2[i] = p_mul(alpha, p_bc(gw[3 + i]));
            E3[i] = p_mul(beta, p_bc(gw[6 + i]));
            a[i]  = p_sub(S[q1i][i], S[q0i][i]);
            b[i]  = p_sub(S[q2i][i], S[q0i][i]);
            D[i]  = p_add(p_add(Dq[q0i][i], Dq[q1i][i]), Dq[q2i][i]);
        }
        f2 gd[3], h[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) gd[i] = p_fma(E3[i], D[i], p_fma(E2[i], b[i], p_mul(E1[i], a[i])));
        // h[k] for the pair (i, j) = (0,1), (0,2), (1,2)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const int i = k == 2 ? 1 : 0, j = k == 0 ? 1 : 2;
            f2        t = p_mul(E1[i], a[j]);
            t           = p_fma(E1[j], a[i], t);
            t           = p_fma(E2[i], b[j], t);
            t           = p_fma(E2[j], b[i], t);
            t           = p_fma(E3[i], D[j], t);
            h[k]        = p_fma(E3[j], D[i], t);
        }
        const f2 tr  = p_add(p_add(gd[0], gd[1]), gd[2]);
        const f2 nkd = p_mul(kw, p_mul(p_bc(-2.0f / 3.0f), tr));
        const f2 k2  = p_add(kw, kw);
        const f2 s00 = p_fma(k2, gd[0], nkd), s11 = p_fma(k2, gd[1], nkd), s22 = p_fma(k2, gd[2], nkd);
        const f2 s01 = p_mul(kw, h[0]), s02 = p_mul(kw, h[1]), s12 = p_mul(kw, h[2]);
        // sigma E for E = E1, E2, E3 (sigma symmetric)
        auto sig = [&](const f2 (&E)[3], f2 (&o)[3]) {
            o[0] = p_fma(s02, E[2], p_fma(s01, E[1], p_mul(s00, E[0])));
            o[1] = p_fma(s12, E[2], p_fma(s11, E[1], p_mul(s01, E[0])));
            o[2] = p_fma(s22, E[2], p_fma(s12, E[1], p_mul(s02, E[0])));
        };
        sig(E1, v1w[w]);
        sig(E2, v2w[w]);
        sig(E3, wvw[w]);
    }
    // corner 0: wedge 0 m=0; corner 3: wedge 1 m=0; corner 1: w0 m=1 + w1 m=2;
    // corner 2: w0 m=2 + w1 m=1 (wedge_corner(1, m) = 3 - m)
    const f2 m1 = make_float2(-1.0f, -1.0f);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const f2 v120 = p_add(v1w[0][c], v2w[0][c]);
        const f2 v121 = p_add(v1w[1][c], v2w[1][c]);
        const f2 rad  = p_add(wvw[0][c], wvw[1][c]);
        const f2 lat1 = p_add(v1w[0][c], v2w[1][c]);
        const f2 lat2 = p_add(v2w[0][c], v1w[1][c]);
        out[0][0][c]  = p_mul(p_add(v120, wvw[0][c]), m1);
        out[0][1][c]  = p_sub(wvw[0][c], v120);
        out[3][0][c]  = p_mul(p_add(v121, wvw[1][c]), m1);
        out[3][1][c]  = p_sub(wvw[1][c], v121);
        out[1][0][c]  = p_sub(lat1, rad);
        out[1][1][c]  = p_add(lat1, rad);
        out[2][0][c]  = p_sub(lat2, rad);
        out[2][1][c]  = p_add(lat2, rad);
    }
}

// Packed FP32 pairs for the interior arithmetic: FP32, an even number of
// radial cells per lane, apply mode (the diagonal mode stays scalar).
template <typename T, int CPL, bool DIAG>
inline constexpr bool kPackedPairs = std::is_same<T, float>::value && (CPL % 2 == 0) && !DIAG;

template <typename T>
struct EddArgs {
    int      nl, nr;
    const T* coords;
    const T* radii;
    const T* k;    // nodal coefficient or nullptr
    const T* kq0;  // per-cell coefficient or nullptr
    const T* src[3];
    T*       dst[3];
    int      bc_cmb, bc_surf;
    int      add;
    int      ty, cx;
    int*     err;
};

template <typename T>
struct SmemLayout {
    size_t   bar_off, ring_off, geo_off, nrm_off, bco_off, xch_off, total;
    uint32_t rowcap;  // bytes per field per row buffer (16-aligned)
};

template <typename T, int CPL>
__host__ __device__ inline SmemLayout<T> edd_smem_layout(int nr, int ty, int cx, int nfields)
{
    SmemLayout<T> L;
    L.bar_off       = 0;  // 3 mbarriers, then the element offsets of the staged rows (3 slots x 4 fields, int)
    L.rowcap        = static_cast<uint32_t>(((static_cast<size_t>(ty + 2) * nr * sizeof(T) + 16) + 15) / 16 * 16);
    L.ring_off      = 128;
    L.geo_off       = L.ring_off + static_cast<size_t>(3) * nfields * L.rowcap;
    L.nrm_off       = L.geo_off + static_cast<size_t>(ty + 1) * (cx + 1) * 20 * sizeof(T);
    L.bco_off       = L.nrm_off + static_cast<size_t>(ty + 1) * (cx + 1) * 12 * sizeof(T);
    L.xch_off       = L.bco_off + static_cast<size_t>(ty + 1) * (cx + 1) * 36 * sizeof(T);
    L.xch_off       = (L.xch_off + 15) / 16 * 16;
    L.total         = L.xch_off + static_cast<size_t>(2) * (ty + 1) * 32 * 3 * (CPL + 1) * sizeof(T);
    return L;
}

template <typename T, int CPL, bool DIAG>
__global__ void __launch_bounds__(32 * MaxWarps<T>::value) epsdivdiv_kernel(EddArgs<T> A)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int nl = A.nl, nr = A.nr;
    const int ty = A.ty, cx = A.cx;
    const int lane = threadIdx.x, w = threadIdx.y, nwarps = ty + 1;
    const int d  = blockIdx.z;
    const int y0 = blockIdx.x * ty;
    const int xs = blockIdx.y * cx;
    const int yc = y0 - 1 + w;  // cell strip of this warp
    const bool q0 = A.kq0 != nullptr;
    const int  nfields = q0 ? 3 : 4;

    const SmemLayout<T> L   = edd_smem_layout<T, CPL>(nr, ty, cx, nfields);
    uint64_t*           bar = reinterpret_cast<uint64_t*>(smem + L.bar_off);
    int*                row_off = reinterpret_cast<int*>(smem + L.bar_off + 32);  // [slot][field]
    unsigned char*      ring = smem + L.ring_off;
    T*                  geo  = reinterpret_cast<T*>(smem + L.geo_off);
    T*                  nrms = reinterpret_cast<T*>(smem + L.nrm_off);
    T*                  bcof = reinterpret_cast<T*>(smem + L.bco_off);
    T*                  xch  = reinterpret_cast<T*>(smem + L.xch_off);

    const int ylo    = max(y0 - 1, 0);
    const int yhi    = min(y0 + ty, nl - 1);
    const int ncols  = yhi - ylo + 1;
    const int nrows  = cx + 2;  // node rows xs-1 .. xs+cx
    const int nsteps = cx + 1;  // cell columns xs-1 .. xs+cx-1
    const T*  fields[4] = {A.src[0], A.src[1], A.src[2], A.k};

    // The issuing thread records, per ring slot and field, the element offset (0..15 bytes / sizeof(T)) of the
    // first staged element in the bulk-copied buffer (each field may sit at a different alignment); the
    // mbarrier's release / acquire makes it visible with the row.
    auto issue_row = [&](int i) {
        const int xr   = xs - 1 + i;
        const int slot = i % 3;
        if (xr < 0 || xr >= nl) {
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(&bar[slot])) : "memory");
            return;
        }
        const int64_t e0    = node_index(nl, nr, d, xr, ylo, 0);
        uint32_t      total = 0;
        uint32_t      bytes[4];
        const T*      srcp[4];
        for (int f = 0; f < nfields; ++f) {
            const uint64_t a   = reinterpret_cast<uint64_t>(fields[f] + e0);
            const uint64_t al  = a & ~uint64_t(15);
            const uint32_t off = static_cast<uint32_t>(a - al);
            bytes[f]           = (off + static_cast<uint32_t>(ncols) * nr * sizeof(T) + 15u) & ~15u;
            srcp[f]            = reinterpret_cast<const T*>(al);
            row_off[slot * 4 + f] = static_cast<int>(off / sizeof(T));
            total += bytes[f];
        }
        mbar_arrive_expect_tx(&bar[slot], total);
        for (int f = 0; f < nfields; ++f)
            bulk_copy_g2s(ring + (static_cast<size_t>(slot) * nfields + f) * L.rowcap, srcp[f], bytes[f], &bar[slot]);
    };

    if (w == 0 && lane == 0) {
        for (int s = 0; s < 3; ++s) mbar_init(&bar[s], 1);
        fence_barrier_init();
    }
    __syncthreads();
    int rows_issued = 0;  // meaningful on the issuing thread only
    if (w == 0 && lane == 0) {
        for (int i = 0; i < 3 && i < nrows; ++i) {
            issue_row(i);
            ++rows_issued;
        }
    }

    // Lateral geometry (and corner normals) of this strip's cells for the
    // chunk, one cell per lane.
    const bool strip_ok = yc >= 0 && yc < nl - 1;
    const bool has_fs   = (A.bc_cmb == 2) || (A.bc_surf == 2);
    for (int i = lane; i < nsteps; i += 32) {
        const int x  = xs - 1 + i;
        T*        g  = geo + (static_cast<size_t>(w) * (cx + 1) + i) * 20;
        T*        nv = nrms + (static_cast<size_t>(w) * (cx + 1) + i) * 12;
        if (strip_ok && x >= 0 && x < nl - 1) {
            column_geometry<T>(A.coords, nl, d, x, yc, g);
            if (has_fs)
                for (int q = 0; q < 4; ++q) {
                    const T* c  = A.coords + node_index(nl, 1, d, x + (q & 1), yc + (q >> 1), 0) * 3;
                    const T  in = T(1) / sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
                    for (int k = 0; k < 3; ++k) nv[q * 3 + k] = c[k] * in;
                }
            // boundary coefficients of the bottom (CMB) and top (surface) cells
            for (int side = 0; side < 2; ++side) {
                const int bc = side == 0 ? A.bc_cmb : A.bc_surf;
                if (bc != 1 && bc != 2) continue;
                const int rc = side == 0 ? 0 : nr - 2;
                const T   r0 = A.radii[rc], r1 = A.radii[rc + 1];
                const T   rm = T(0.5) * (r0 + r1), hdr = T(0.5) * (r1 - r0);
                boundary_coefficients<T>(g, T(0.5) / rm, T(1) / (T(6) * hdr), rm * rm * hdr * (q0 ? T(1) : T(1) / T(6)),
                                         side, bc, nv, bcof + ((static_cast<size_t>(w) * (cx + 1) + i) * 2 + side) * 18);
            }
        } else {
            for (int v = 0; v < 20; ++v) g[v] = T(0);
        }
    }

    // Per-lane radial constants.
    T   alpha[CPL], beta[CPL], dfac[CPL];
    int cbc[CPL][2];
#pragma unroll
    for (int j = 0; j < CPL; ++j) {
        const int c = lane + 32 * j;
        if (c < nr - 1) {
            const T r0 = A.radii[c], r1 = A.radii[c + 1];
            const T rm = T(0.5) * (r0 + r1), hdr = T(0.5) * (r1 - r0);
            alpha[j]   = T(0.5) / rm;
            beta[j]    = T(1) / (T(6) * hdr);
            dfac[j]    = rm * rm * hdr * (q0 ? T(1) : T(1) / T(6));
        } else {
            alpha[j] = beta[j] = dfac[j] = T(0);
        }
        cbc[j][0] = (c == 0) ? A.bc_cmb : 0;
        cbc[j][1] = (c == nr - 2) ? A.bc_surf : 0;
    }
    // Radial mapping: lane l holds cells l + 32 j (j < CPL), so shared-memory
    // reads and global stores are consecutive across lanes. The top node nr-1
    // is the extra node of the lane/iteration holding cell nr-2.
    const int lane_top = (nr - 2) % 32;
    const int j_top    = (nr - 2) / 32;

    T xcarry[2][CPL + 1][3];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int j = 0; j <= CPL; ++j)
#pragma unroll
            for (int c = 0; c < 3; ++c) xcarry[a][j][c] = T(0);

    __syncwarp();

    bool ok        = true;
    int  rows_done = 0;  // rows this thread has seen land, in order
    for (int i = 0; i < nsteps; ++i) {
        const int x = xs - 1 + i;
        // rows i and i + 1 must be resident
        if (ok && i == 0) {
            ok = mbar_wait_bounded(&bar[0], 0);
            rows_done += ok ? 1 : 0;
        }
        if (ok) {
            ok = mbar_wait_bounded(&bar[(i + 1) % 3], ((i + 1) / 3) & 1);
            rows_done += ok ? 1 : 0;
        }
        if (!ok) report_error(A.err, kDevMbarrierTimeout);
        int offA[4], offB[4];
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            offA[f] = (f < nfields && x >= 0 && x < nl) ? row_off[(i % 3) * 4 + f] : 0;
            offB[f] = (f < nfields && x + 1 >= 0 && x + 1 < nl) ? row_off[((i + 1) % 3) * 4 + f] : 0;
        }
        const T*  rowA = reinterpret_cast<const T*>(ring + static_cast<size_t>(i % 3) * nfields * L.rowcap);
        const T*  rowB = reinterpret_cast<const T*>(ring + static_cast<size_t>((i + 1) % 3) * nfields * L.rowcap);
        const bool cell_col_ok = strip_ok && x >= 0 && x < nl - 1;
        const T*   g           = geo + (static_cast<size_t>(w) * (cx + 1) + i) * 20;

        const T* nrm_col = nrms + (static_cast<size_t>(w) * (cx + 1) + i) * 12;

        // Radial sums (node rc = bottom of cell rc + top of cell rc - 1) feed the
        // x carry and the y exchange as soon as a node is complete.
        T* slot_w = xch + (static_cast<size_t>(i & 1) * nwarps + w) * 3 * (CPL + 1) * 32 + lane;
        T  keep[CPL + 1][3];
        T  carry31[4][3];  // top of cell 32 j - 1 (lane 31, previous j)
        auto finish_node = [&](int j, const T (&nv)[4][3]) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                keep[j][c]                = nv[0][c] + xcarry[0][j][c];
                slot_w[(j * 3 + c) * 32] = nv[2][c] + xcarry[1][j][c];
                xcarry[0][j][c]           = nv[1][c];
                xcarry[1][j][c]           = nv[3][c];
            }
        };

        // Staged inputs of cell rc of this column (the caller checks validity).
        auto load_cell = [&](int rc, T (&u)[4][2][3], T (&ks)[4], T& kcell) {
            const int e0 = (yc - ylo) * nr + rc;      // corners dy = 0
            const int e1 = (yc + 1 - ylo) * nr + rc;  // corners dy = 1
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const unsigned char* row = reinterpret_cast<const unsigned char*>((q & 1) ? rowB : rowA);
                const int*           off = (q & 1) ? offB : offA;
                const int            e   = (q >> 1) ? e1 : e0;
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const T* fr = reinterpret_cast<const T*>(row + static_cast<size_t>(c) * L.rowcap) + off[c];
                    u[q][0][c]  = fr[e];
                    u[q][1][c]  = fr[e + 1];
                }
                if (!q0) {
                    const T* kr = reinterpret_cast<const T*>(row + static_cast<size_t>(3) * L.rowcap) + off[3];
                    ks[q]       = kr[e] + kr[e + 1];
                } else {
                    ks[q] = T(0);
                }
            }
            kcell = q0 ? A.kq0[node_index(nl - 1, nr - 1, d, x, yc, rc)] : T(0);
        };
        // Unmodified side-s values of cell rc (boundary rows).
        auto load_raw = [&](int rc, int side, T (&raw)[4][3]) {
            const int e0 = (yc - ylo) * nr + rc + side;
            const int e1 = (yc + 1 - ylo) * nr + rc + side;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const unsigned char* row = reinterpret_cast<const unsigned char*>((q & 1) ? rowB : rowA);
                const int*           off = (q & 1) ? offB : offA;
                const int            e   = (q >> 1) ? e1 : e0;
#pragma unroll
                for (int c = 0; c < 3; ++c)
                    raw[q][c] = reinterpret_cast<const T*>(row + static_cast<size_t>(c) * L.rowcap)[off[c] + e];
            }
        };
        const T* bco_col = bcof + (static_cast<size_t>(w) * (cx + 1) + i) * 2 * 18;

        // Scalar path: one cell (all modes).
        auto scalar_cell = [&](int j, T (&out)[4][2][3]) {
            const int rc = lane + 32 * j;
            if (ok && cell_col_ok && rc < nr - 1) {
                T u[4][2][3], ks[4], kcell;
                load_cell(rc, u, ks, kcell);
                if (DIAG) {
                    const int bcs[2] = {cbc[j][0], cbc[j][1]};
                    T         nrm[4][3];
#pragma unroll
                    for (int q = 0; q < 4; ++q)
#pragma unroll
                        for (int c = 0; c < 3; ++c) {
                            nrm[q][c] = has_fs ? nrm_col[q * 3 + c] : T(0);
#pragma unroll
                            for (int sd = 0; sd < 2; ++sd) out[q][sd][c] = T(0);
                        }
                    cell_apply<T, true>(u, ks, kcell, q0, g, alpha[j], beta[j], dfac[j], bcs, nrm, out);
                } else {
                    // boundary cells: only lane 0 (CMB, j = 0) and lane_top (surface, last j)
                    const bool b0 = cbc[j][0] != 0;
                    const bool b1 = cbc[j][1] != 0;
                    T          un0[4], un1[4];
                    if (b0) side_inputs<T>(u, 0, cbc[j][0], nrm_col, un0);
                    if (b1) side_inputs<T>(u, 1, cbc[j][1], nrm_col, un1);
                    hex_interior<T>(u, ks, kcell, q0, g, alpha[j], beta[j], dfac[j], out);
#pragma unroll
                    for (int side = 0; side < 2; ++side) {
                        if (!(side == 0 ? b0 : b1)) continue;
                        T raw[4][3];
                        load_raw(rc, side, raw);
                        side_outputs<T>(out, side, side == 0 ? cbc[j][0] : cbc[j][1], ks, kcell, q0,
                                        bco_col + side * 18, nrm_col, raw, side == 0 ? un0 : un1);
                    }
                }
            } else {
#pragma unroll
                for (int q = 0; q < 4; ++q)
#pragma unroll
                    for (int sd = 0; sd < 2; ++sd)
#pragma unroll
                        for (int c = 0; c < 3; ++c) out[q][sd][c] = T(0);
            }
        };

        // Radial sums of cell j's outputs into node values.
        auto combine = [&](int j, const T (&out)[4][2][3]) {
            T nv[4][3], top[4][3];
#pragma unroll
            for (int q = 0; q < 4; ++q)
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    top[q][c]     = out[q][1][c];
                    const T up    = shfl_up(top[q][c], 1);
                    const T below = lane > 0 ? up : (j > 0 ? carry31[q][c] : T(0));
                    nv[q][c]      = out[q][0][c] + below;
                }
            finish_node(j, nv);
            if (j == j_top) finish_node(CPL, top);
            if (j + 1 < CPL) {
#pragma unroll
                for (int q = 0; q < 4; ++q)
#pragma unroll
                    for (int c = 0; c < 3; ++c) carry31[q][c] = __shfl_sync(0xffffffffu, top[q][c], 31);
            }
        };

        if constexpr (kPackedPairs<T, CPL, DIAG>) {
            // FP32: cells (j, j + 1) of the lane as one packed pair
#pragma unroll
            for (int j = 0; j < CPL; j += 2) {
                const int  rcA = lane + 32 * j, rcB = rcA + 32;
                const bool vA  = ok && cell_col_ok && rcA < nr - 1;
                const bool vB  = ok && cell_col_ok && rcB < nr - 1;
                T          uA[4][2][3], uB[4][2][3], ksA[4], ksB[4], kA = T(0), kB = T(0);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    ksA[q] = ksB[q] = T(0);
#pragma unroll
                    for (int sd = 0; sd < 2; ++sd)
#pragma unroll
                        for (int c = 0; c < 3; ++c) uA[q][sd][c] = uB[q][sd][c] = T(0);
                }
                if (vA) load_cell(rcA, uA, ksA, kA);
                if (vB) load_cell(rcB, uB, ksB, kB);
                // boundary cells: CMB is cell 0 (lane 0, j = 0), the surface cell nr - 2
                const bool b0A = vA && cbc[j][0] != 0, b1A = vA && cbc[j][1] != 0;
                const bool b0B = vB && cbc[j + 1][0] != 0, b1B = vB && cbc[j + 1][1] != 0;
                T          un0A[4], un1A[4], un0B[4], un1B[4];
                if (b0A) side_inputs<T>(uA, 0, cbc[j][0], nrm_col, un0A);
                if (b1A) side_inputs<T>(uA, 1, cbc[j][1], nrm_col, un1A);
                if (b0B) side_inputs<T>(uB, 0, cbc[j + 1][0], nrm_col, un0B);
                if (b1B) side_inputs<T>(uB, 1, cbc[j + 1][1], nrm_col, un1B);
                f2 u2[4][2][3], ks2[4], o2[4][2][3];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    ks2[q] = make_float2(ksA[q], ksB[q]);
#pragma unroll
                    for (int sd = 0; sd < 2; ++sd)
#pragma unroll
                        for (int c = 0; c < 3; ++c) u2[q][sd][c] = make_float2(uA[q][sd][c], uB[q][sd][c]);
                }
                hex_interior_x2(u2, ks2, make_float2(kA, kB), q0, reinterpret_cast<const float*>(g),
                                make_float2(alpha[j], alpha[j + 1]), make_float2(beta[j], beta[j + 1]),
                                make_float2(dfac[j], dfac[j + 1]), o2);
                T oA[4][2][3], oB[4][2][3];
#pragma unroll
                for (int q = 0; q < 4; ++q)
#pragma unroll
                    for (int sd = 0; sd < 2; ++sd)
#pragma unroll
                        for (int c = 0; c < 3; ++c) {
                            oA[q][sd][c] = o2[q][sd][c].x;
                            oB[q][sd][c] = o2[q][sd][c].y;
                        }
                if (b0A || b1A) {
#pragma unroll
                    for (int side = 0; side < 2; ++side) {
                        if (!(side == 0 ? b0A : b1A)) continue;
                        T raw[4][3];
                        load_raw(rcA, side, raw);
                        side_outputs<T>(oA, side, cbc[j][side], ksA, kA, q0, bco_col + side * 18, nrm_col, raw,
                                        side == 0 ? un0A : un1A);
                    }
                }
                if (b0B || b1B) {
#pragma unroll
                    for (int side = 0; side < 2; ++side) {
                        if (!(side == 0 ? b0B : b1B)) continue;
                        T raw[4][3];
                        load_raw(rcB, side, raw);
                        side_outputs<T>(oB, side, cbc[j + 1][side], ksB, kB, q0, bco_col + side * 18, nrm_col, raw,
                                        side == 0 ? un0B : un1B);
                    }
                }
                combine(j, oA);
                combine(j + 1, oB);
            }
        } else {
#pragma unroll
            for (int j = 0; j < CPL; ++j) {
                T out[4][2][3];
                scalar_cell(j, out);
                combine(j, out);
            }
        }
        __syncthreads();
        if (w == 0 && lane == 0 && i + 3 < nrows) {
            issue_row(i + 3);
            ++rows_issued;
        }

        const int yn = yc;  // node line owned by warp w (w >= 1)
        if (ok && w >= 1 && i >= 1 && x < nl && yn < nl) {
            const T*  slot_p = xch + (static_cast<size_t>(i & 1) * nwarps + (w - 1)) * 3 * (CPL + 1) * 32 + lane;
            const int obase  = ((d * nl + x) * nl + yn) * nr;  // 32-bit: the host limits a level to 2^31 nodes
#pragma unroll
            for (int j = 0; j <= CPL; ++j) {
                const int rn = (j < CPL) ? lane + 32 * j : nr - 1;
                const bool own = (j < CPL) ? (rn < nr - 1) : (lane == lane_top);
                if (!own) continue;
                const int id = obase + rn;
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const T v = keep[j][c] + slot_p[(j * 3 + c) * 32];
                    if (A.add)
                        A.dst[c][id] += v;
                    else
                        A.dst[c][id] = v;
                }
            }
        }
    }
    // After a timeout the issuing thread still waits (bounded) for every bulk
    // copy it issued, so no copy lands in shared memory after the CTA retires.
    if (w == 0 && lane == 0) {
        for (int r = rows_done; r < rows_issued; ++r) (void)mbar_wait_bounded(&bar[r % 3], (r / 3) & 1, 100000000ull);
    }
}

template <typename T, int CPL, bool DIAG>
int launch_cfg(EddArgs<T> a, int nfields, cudaStream_t st)
{
    constexpr size_t kSmemLimit = 227 * 1024;
    SmemLayout<T>    L          = edd_smem_layout<T, CPL>(a.nr, a.ty, a.cx, nfields);
    while (L.total > kSmemLimit && a.cx > 1) {
        a.cx = (a.cx + 1) / 2;
        L    = edd_smem_layout<T, CPL>(a.nr, a.ty, a.cx, nfields);
    }
    if (L.total > kSmemLimit) return -5;
    auto k = epsdivdiv_kernel<T, CPL, DIAG>;
    // the dynamic shared-memory limit is a per-device attribute of the kernel:
    // raise it once per device, only upwards; the check, the attribute call
    // and the record happen under one lock so racing threads cannot lower it
    static std::mutex mu;
    static size_t     configured[kMaxDevices];
    int               dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return -1;
    {
        std::lock_guard<std::mutex> lock(mu);
        if (L.total > configured[dev]) {
            if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(L.total)) !=
                cudaSuccess)
                return -1;
            configured[dev] = L.total;
        }
    }
    const int nl = a.nl;
    dim3      grid((nl + a.ty - 1) / a.ty, (nl + a.cx - 1) / a.cx, 10);
    dim3      block(32, a.ty + 1);
    k<<<grid, block, L.total, st>>>(a);
    note_launch();
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

template <typename T>
int launch(const EddArgs<T>& a, bool diag, cudaStream_t st)
{
    const int cells = a.nr - 1;
    const int nf    = a.kq0 ? 3 : 4;
    if (cells <= 32) return diag ? launch_cfg<T, 1, true>(a, nf, st) : launch_cfg<T, 1, false>(a, nf, st);
    if (cells <= 64) return diag ? launch_cfg<T, 2, true>(a, nf, st) : launch_cfg<T, 2, false>(a, nf, st);
    if (cells <= 128) return diag ? launch_cfg<T, 4, true>(a, nf, st) : launch_cfg<T, 4, false>(a, nf, st);
    return -3;
}

}  // namespace

template <typename T>
int epsdivdiv_apply(const EddLaunch<T>& p, cudaStream_t stream)
{
    EddArgs<T> a;
    a.nl     = p.nl;
    a.nr     = p.nr;
    a.coords = p.coords;
    a.radii  = p.radii;
    a.k      = p.k;
    a.kq0    = p.kq0;
    for (int c = 0; c < 3; ++c) {
        a.src[c] = p.src[c];
        a.dst[c] = p.dst[c];
    }
    a.bc_cmb  = p.bc_cmb;
    a.bc_surf = p.bc_surf;
    a.add     = p.add;
    a.err     = p.err;
    // tile shape: TY node lines per CTA (TY + 1 warps), CX node rows per x chunk
    a.ty = p.tile_y > 0 ? p.tile_y : std::min(MaxWarps<T>::value - 1, p.nl);
    if (p.chunk_x > 0) {
        a.cx = p.chunk_x;
    } else {
        // One CTA per SM: pick the x-chunk that minimises waves x steps per CTA.
        static std::atomic<int> sm_count[kMaxDevices];
        int                     dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return -1;
        int sms = sm_count[dev].load(std::memory_order_relaxed);
        if (sms == 0) {
            if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
            sm_count[dev].store(sms, std::memory_order_relaxed);
        }
        const int ytiles = (p.nl + a.ty - 1) / a.ty;
        long      best   = -1;
        for (int cx = 4; cx <= std::max(4, p.nl); ++cx) {
            const long ctas  = 10L * ytiles * ((p.nl + cx - 1) / cx);
            const long waves = (ctas + sms - 1) / sms;
            const long cost  = waves * (cx + 1);
            if (best < 0 || cost < best || (cost == best && cx > a.cx)) {
                best = cost;
                a.cx = cx;
            }
        }
    }
    if (a.ty + 1 > MaxWarps<T>::value) return -4;
    if (10LL * p.nl * p.nl * p.nr >= (1LL << 31)) return -6;  // the kernel indexes nodes in 32 bits
    return launch<T>(a, p.diagonal, stream);
}

template int epsdivdiv_apply<double>(const EddLaunch<double>&, cudaStream_t);
template int epsdivdiv_apply<float>(const EddLaunch<float>&, cudaStream_t);

}  // namespace tn
