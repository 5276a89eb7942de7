// Galerkin coarse approximation (GCA) of the epsilon-div-div operator and the
// stored-matrix apply (FP64 build, FP64/FP32 apply).
//
// Build (TwoGridGCA, src/terra/linalg/solvers/gca/gca.hpp:154-530): for every
// coarse hex and each of its 8 fine hexes x 2 wedges, A_c[t] += P^T A_f P with
// P the 6x6 constant-weight interpolation from the coarse wedge's nodes to the
// fine wedge's nodes (vectorised block-diagonally over the 3 components) and t
// the coarse wedge containing the fine wedge. The fine matrices are the
// on-the-fly Neumann element matrices of the finest level
// (assemble_local_matrix, epsilon_divdiv_kerngen.hpp:2315-2392) or the stored
// GCA matrices of the next finer level. P follows gca.hpp:204-383 exactly,
// including its radial bracket r_bot = r_fine/2 (r_fine/2 - 1 on the outer
// shell), which for fine nodes on the top plane of a coarse hex points the
// lateral weights at the coarse wedge's bottom nodes.
//
// One CTA of 18 x 18 threads per coarse hex; thread (i, j) owns entry (i, j) of
// both coarse wedge matrices. Matrices are stored packed-symmetric (171 values
// per wedge, upper triangle, dimension-wise ordering index = node + 6 dim) as
// value-major arrays [wedge * 171 + p][cell] so that consecutive cells are
// consecutive in memory.
//
// Boundary conditions are applied at coarse-apply time in the reference
// (slow path, epsilon_divdiv_kerngen.hpp:1013-1242). Here they are baked into a
// copy of the matrices once: Dirichlet -> mask off-diagonal couplings of
// boundary-node rows / columns; free-slip -> R^T (M o (R A R^T)) R with R the
// normal-tangential frames of the boundary nodes and M masking the normal
// component. The apply is then a plain symmetric matvec; the reference's
// diagonal mode (rotated diagonal on free-slip nodes) has its own kernel.
#include <mutex>

#include "tn_device.cuh"
#include "tn_kernels.hpp"
#include "tn_wedge_math.cuh"

namespace tn {
namespace {

constexpr int kN = 18, kPack = 171;

__host__ __device__ constexpr int woff(int w, int n, int k)
{
    constexpr int t[2][6][3] = {{{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {0, 1, 1}},
                                {{1, 1, 0}, {0, 1, 0}, {1, 0, 0}, {1, 1, 1}, {0, 1, 1}, {1, 0, 1}}};
    return t[w][n][k];
}

__host__ __device__ __forceinline__ int pidx(int i, int j)
{
    if (i > j) {
        const int t = i;
        i           = j;
        j           = t;
    }
    return i * (2 * kN - i + 1) / 2 + (j - i);
}

// prolongation_constant_weight (grid_transfer_constant.hpp:24-89)
__device__ __forceinline__ double pweight(int xf, int yf, int rf, int xc, int yc, int rc)
{
    const int dx = xf - 2 * xc, dy = yf - 2 * yc, dr = rf - 2 * rc;
    double    lat = 0.0;
    if (dx == 0 && dy == 0)
        lat = 1.0;
    else if (dy == 0 && (dx == 1 || dx == -1))
        lat = 0.5;
    else if (dx == 0 && (dy == 1 || dy == -1))
        lat = 0.5;
    else if ((dx == -1 && dy == 1) || (dx == 1 && dy == -1))
        lat = 0.5;
    if (dr == 0) return lat;
    if (dr == 1 || dr == -1) return 0.5 * lat;
    return 0.0;
}

// Row fl of the interpolation matrix P[fine node][coarse node] of fine wedge (fx, fy, fr, w) (gca.hpp:204-383):
// InterpolationMode::Constant, or InterpolationMode::Linear when linw (the fine level's linear-transfer weights,
// two per node: prolongation_linear_weights) is given.
__device__ void interp_row(int d, int fx, int fy, int fr, int w, int fl, int nlf, int nrf, const double* linw,
                           double* row)
{
    for (int b = 0; b < 6; ++b) row[b] = 0.0;
    const int ix = fx + woff(w, fl, 0), iy = fy + woff(w, fl, 1), ir = fr + woff(w, fl, 2);
    if (ix % 2 == 0 && iy % 2 == 0 && ir % 2 == 0) {
        row[fl] = 1.0;
        return;
    }
    const int rb = ir < nrf - 1 ? ir / 2 : ir / 2 - 1, rt = rb + 1;
    double    lw0 = 0.0, lw1 = 0.0;
    if (linw) {
        const int64_t fi = node_index(nlf, nrf, d, ix, iy, ir);
        lw0              = linw[2 * fi];
        lw1              = linw[2 * fi + 1];
    }
    if (ix % 2 == 0 && iy % 2 == 0) {
        const int a = fl % 3;  // lateral index of the fine node == coarse node
        row[a]      = linw ? lw0 : 0.5;
        row[a + 3]  = linw ? lw1 : 0.5;
        return;
    }
    int x0, x1, y0, y1, c0, c1, c2, c3;
    if (ix % 2 == 0) {
        x0 = ix / 2, x1 = ix / 2, y0 = iy / 2, y1 = iy / 2 + 1;
        c0 = 0, c1 = 2, c2 = 3, c3 = 5;
    } else if (iy % 2 == 0) {
        x0 = ix / 2, x1 = ix / 2 + 1, y0 = iy / 2, y1 = iy / 2;
        c0 = 0, c1 = 1, c2 = 3, c3 = 4;
    } else {
        x0 = ix / 2 + 1, x1 = ix / 2, y0 = iy / 2, y1 = iy / 2 + 1;
        c0 = 1, c1 = 2, c2 = 4, c3 = 5;
    }
    if (linw) {
        row[c0] = lw0;
        row[c1] = lw0;
        row[c2] = lw1;
        row[c3] = lw1;
        return;
    }
    row[c0] = pweight(ix, iy, ir, x0, y0, rb);
    row[c1] = pweight(ix, iy, ir, x1, y1, rb);
    row[c2] = pweight(ix, iy, ir, x0, y0, rt);
    row[c3] = pweight(ix, iy, ir, x1, y1, rt);
}

__device__ void interp_matrix(int d, int fx, int fy, int fr, int w, int nlf, int nrf, const double* linw,
                              double (&P)[6][6])
{
    for (int fl = 0; fl < 6; ++fl) interp_row(d, fx, fy, fr, w, fl, nlf, nrf, linw, P[fl]);
}

// coarse wedge receiving fine hex h (x + 2 y + 4 r shift order of gca.hpp:176-185) wedge w
__host__ __device__ __forceinline__ int target_wedge(int h, int w)
{
    const int hl = h & 3;  // lateral position in the coarse hex: 0 (0,0) 1 (1,0) 2 (0,1) 3 (1,1)
    if (w == 0) return hl == 3 ? 1 : 0;
    return hl == 0 ? 0 : 1;
}

struct GcaBuildArgs {
    int           nlf = 0, nrf = 0;     // fine level dims
    const double* coords    = nullptr;  // fine coords
    const double* radii     = nullptr;  // fine radii
    const double* k         = nullptr;  // fine nodal coefficient (on-the-fly matrices) or nullptr
    const double* kq0       = nullptr;  // fine cell coefficient or nullptr
    const double* fine_mats = nullptr;  // stored fine matrices [342][fine_stride] or nullptr
    double*       out       = nullptr;  // coarse matrices [342][nout]
    const double* linw      = nullptr;  // fine linear-transfer weights (linear interpolation) or nullptr (constant)
    // selective storage (LocalMatrixStorage, local_matrix_storage.hpp:136-165): the coarse cells to build, slot s
    // of out holding cells[s] (nullptr: every cell, slot = cell), and the slot of each fine cell in fine_mats
    // (nullptr: slot = cell). A fine cell without a slot reports kDevBadLaunch to err and reads as zero.
    const int* cells       = nullptr;
    int        nout        = 0;
    const int* fine_slot   = nullptr;
    int        fine_stride = 0;
    int*       err         = nullptr;
};

// (d, x, y, r) of a cell index of a level with nl lateral and nr radial nodes
__device__ __forceinline__ void decode_cell(int cell, int nl, int nr, int& d, int& x, int& y, int& r)
{
    r     = cell % (nr - 1);
    int t = cell / (nr - 1);
    y     = t % (nl - 1);
    t /= (nl - 1);
    x = t % (nl - 1);
    d = t / (nl - 1);
}

// stored value p (0..341) of fine cell (d, x, y, r)
__device__ __forceinline__ double fine_value(const GcaBuildArgs& A, int d, int x, int y, int r, int p)
{
    const int fc   = static_cast<int>(node_index(A.nlf - 1, A.nrf - 1, d, x, y, r));
    const int slot = A.fine_slot ? A.fine_slot[fc] : fc;
    if (slot < 0) {
        report_error(A.err, kDevBadLaunch);
        return 0.0;
    }
    return A.fine_mats[static_cast<int64_t>(p) * A.fine_stride + slot];
}

// Fine wedge matrix of (d, fx, fy, fr, w) into Af (dimension-wise ordering),
// either assembled on the fly or read from stored matrices. Called by all
// 18 x 18 threads of the CTA; ends with the matrix visible to all of them.
__device__ void fine_wedge_factors(const GcaBuildArgs& A, int d, int fx, int fy, int fr, int w, double (&G)[6][3],
                                   double& kwJ);

__device__ void load_fine_matrix(const GcaBuildArgs& A, int d, int fx, int fy, int fr, int w, double (&Af)[kN][kN],
                                 double (&G)[6][3], double& kwJ)
{
    const int  tid = threadIdx.x;
    const bool ent = tid < kN * kN;  // threads beyond the 324 entries only take part in the barrier
    const int  i = ent ? tid / kN : 0, j = ent ? tid % kN : 0;
    const int  ni = i % 6, di = i / 6, nj = j % 6, dj = j / 6;
    if (A.fine_mats == nullptr) {
        // element matrix: gradients and k|det J| first
        if (tid == 0) fine_wedge_factors(A, d, fx, fy, fr, w, G, kwJ);
        __syncthreads();
        // A(i,j) = kwJ [delta_{di dj} g_i.g_j + g_i[dj] g_j[di] - 2/3 g_i[di] g_j[dj]]
        const double gij = (di == dj) ? (G[ni][0] * G[nj][0] + G[ni][1] * G[nj][1] + G[ni][2] * G[nj][2]) : 0.0;
        if (ent) Af[i][j] = kwJ * (gij + G[ni][dj] * G[nj][di] - (2.0 / 3.0) * G[ni][di] * G[nj][dj]);
    } else if (ent) {
        Af[i][j] = fine_value(A, d, fx, fy, fr, w * kPack + pidx(i, j));
    }
}

// Gradients g_n (physical) of the six shape functions of fine wedge (d, fx, fy, fr, w) at its centroid and
// the weight kwJ = k(centroid) |det J| of the one-point rule: the factors of the on-the-fly element matrix
// A(i,j) = kwJ [delta_{di dj} g_i.g_j + g_i[dj] g_j[di] - 2/3 g_i[di] g_j[dj]] (load_fine_matrix).
__device__ void fine_wedge_factors(const GcaBuildArgs& A, int d, int fx, int fy, int fr, int w, double (&G)[6][3],
                                   double& kwJ)
{
    const int nlf = A.nlf, nrf = A.nrf;
    double    geo[20];
    column_geometry<double>(A.coords, nlf, d, fx, fy, geo);
    const double  r0 = A.radii[fr], r1 = A.radii[fr + 1];
    const double  rm = 0.5 * (r0 + r1), hdr = 0.5 * (r1 - r0);
    const double  alpha = 0.5 / rm, beta = 1.0 / (6.0 * hdr);
    const double* gw    = geo + 10 * w;
    for (int n = 0; n < 6; ++n) {
        const int    m  = n % 3;
        const double sg = n < 3 ? -1.0 : 1.0;
        for (int c = 0; c < 3; ++c) {
            const double L = m == 0 ? -(gw[c] + gw[3 + c]) : (m == 1 ? gw[c] : gw[3 + c]);
            G[n][c]        = alpha * L + sg * beta * gw[6 + c];
        }
    }
    double kv;
    if (A.kq0) {
        kv = A.kq0[node_index(nlf - 1, nrf - 1, d, fx, fy, fr)];
    } else {
        // shape functions at the centroid (assemble_trial_test_vecs,
        // epsilon_divdiv_kerngen.hpp:2258-2264): lateral 1/3 each, radial 1/2
        const double wlat0 = 1.0 - 1.0 / 3.0 - 1.0 / 3.0, wlat = 1.0 / 3.0;
        kv                 = 0.0;
        for (int n = 0; n < 6; ++n)
            kv += (n % 3 == 0 ? wlat0 : wlat) * 0.5 *
                  A.k[node_index(nlf, nrf, d, fx + woff(w, n, 0), fy + woff(w, n, 1), fr + woff(w, n, 2))];
    }
    kwJ = kv * gw[9] * rm * rm * hdr;
}

// (row, column) of packed entry p of the upper triangle
__device__ __forceinline__ void packed_pair(int p, int& i, int& j)
{
    int a = 0;
    while (p >= kN - a) {
        p -= kN - a;
        ++a;
    }
    i = a;
    j = a + p;
}

// coarse cell of this CTA: slot blockIdx.x of the output, cells[slot] (or slot) on the coarse level
__device__ __forceinline__ bool coarse_cell_of_block(const GcaBuildArgs& A, int& slot, int& d, int& xc, int& yc,
                                                     int& rc)
{
    const int nlc = (A.nlf + 1) / 2, nrc = (A.nrf + 1) / 2;
    slot          = blockIdx.x;
    if (slot >= A.nout) return false;
    decode_cell(A.cells ? A.cells[slot] : slot, nlc, nrc, d, xc, yc, rc);
    return true;
}

// fine hex h (x + 2 y + 4 r shift order of gca.hpp:176-185) of coarse hex (xc, yc, rc)
__device__ __forceinline__ void fine_hex(int h, int xc, int yc, int rc, int& fx, int& fy, int& fr)
{
    fx = 2 * xc + (h & 1);
    fy = 2 * yc + ((h >> 1) & 1);
    fr = 2 * rc + ((h >> 2) & 1);
}

// Plain form, one fine wedge at a time in the reference's order (fine matrix, then P^T A_f P): one CTA of
// 18 x 18 threads per coarse hex, thread (i, j) owns entry (i, j) of both coarse wedge matrices.
__global__ void __launch_bounds__(kN * kN) gca_build_kernel(GcaBuildArgs A)
{
    const int nlf = A.nlf, nrf = A.nrf;
    int       slot, d, xc, yc, rc;
    if (!coarse_cell_of_block(A, slot, d, xc, yc, rc)) return;

    const int tid = threadIdx.x;
    const int i = tid / kN, j = tid % kN;  // matrix entry of this thread
    const int ni = i % 6, di = i / 6, nj = j % 6, dj = j / 6;

    __shared__ double Af[kN][kN];
    __shared__ double Y[kN][kN];
    __shared__ double P[6][6];
    __shared__ double G[6][3];
    __shared__ double kwJ;

    double acc0 = 0.0, acc1 = 0.0;
    for (int h = 0; h < 8; ++h) {
        int fx, fy, fr;
        fine_hex(h, xc, yc, rc, fx, fy, fr);
        for (int w = 0; w < 2; ++w) {
            load_fine_matrix(A, d, fx, fy, fr, w, Af, G, kwJ);
            if (tid == 0) interp_matrix(d, fx, fy, fr, w, nlf, nrf, A.linw, P);
            __syncthreads();
            // Y = A P_vec: P_vec couples equal dimensions only
            double y = 0.0;
            for (int l = 0; l < 6; ++l) y += Af[i][l + 6 * dj] * P[l][nj];
            Y[i][j] = y;
            __syncthreads();
            double v = 0.0;
            for (int kk = 0; kk < 6; ++kk) v += P[kk][ni] * Y[kk + 6 * di][j];
            if (target_wedge(h, w) == 0)
                acc0 += v;
            else
                acc1 += v;
            __syncthreads();
        }
    }
    if (i <= j) {
        A.out[static_cast<int64_t>(0 * kPack + pidx(i, j)) * A.nout + slot] = acc0;
        A.out[static_cast<int64_t>(1 * kPack + pidx(i, j)) * A.nout + slot] = acc1;
    }
}

// Coarse hexes over stored fine matrices: the triple products on the FP64 tensor cores (mma.sync m8n8k4, f64
// in and out). P_vec = I_3 (x) P couples equal dimensions only, so A_c += P_vec^T A_f P_vec splits into nine
// 6 x 6 blocks A_c[di][dj] += P^T A_f[di][dj] P. The CTA first stages all 16 fine wedge matrices (unpacked)
// and their interpolation matrices in shared memory, with one barrier. Warp b of the first nine then owns
// block b = (di, dj) for both coarse wedges, kept in two 8 x 8 accumulator fragments (blocks and P
// zero-padded to 8 x 8); per fine wedge it runs Y = A_f[di][dj] P (two k = 4 steps) and A_c += P^T Y (two
// more), staging Y through its own shared tile to turn the accumulator layout into the B-operand layout, with
// warp-level synchronisation only.
constexpr int kMmaWarps   = 11;  // 352 threads: all stage, warps 0-8 own the nine blocks
constexpr int kMmaThreads = 32 * kMmaWarps;
constexpr int kFineWedges = 16;
constexpr size_t kMmaSmem = sizeof(double) * (kFineWedges * kN * kN + kFineWedges * 36 + 9 * 64);

__device__ __forceinline__ void dmma_8x8x4(double (&d)[2], double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(kMmaThreads) gca_build_mma_kernel(GcaBuildArgs A)
{
    const int nlf = A.nlf, nrf = A.nrf;
    int       slot, d, xc, yc, rc;
    if (!coarse_cell_of_block(A, slot, d, xc, yc, rc)) return;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int b = warp < 9 ? warp : 0, bdi = b / 3, bdj = b % 3;  // block (di, dj) of this warp
    const int fr_row = lane >> 2, fr_col = lane & 3;             // fragment coordinates (PTX m8n8k4 f64)

    extern __shared__ double smem[];
    double(*Af)[kN][kN] = reinterpret_cast<double(*)[kN][kN]>(smem);
    double(*P)[6][6]    = reinterpret_cast<double(*)[6][6]>(smem + kFineWedges * kN * kN);
    double(*Yb)[8][8]   = reinterpret_cast<double(*)[8][8]>(smem + kFineWedges * (kN * kN + 36));

    // fine wedge f = 2 h + w: the 96 rows of the 16 interpolation matrices, one per thread
    if (tid < 6 * kFineWedges) {
        const int f = tid / 6, fl = tid % 6;
        int       fx, fy, fr;
        fine_hex(f >> 1, xc, yc, rc, fx, fy, fr);
        interp_row(d, fx, fy, fr, f & 1, fl, nlf, nrf, A.linw, P[f][fl]);
    }
    for (int e = tid; e < kFineWedges * kPack; e += kMmaThreads) {
        const int f = e / kPack, p = e % kPack;
        int       fx, fy, fr, i, j;
        fine_hex(f >> 1, xc, yc, rc, fx, fy, fr);
        packed_pair(p, i, j);
        const double v = fine_value(A, d, fx, fy, fr, (f & 1) * kPack + p);
        Af[f][i][j]    = v;
        Af[f][j][i]    = v;
    }
    __syncthreads();
    if (warp >= 9) return;

    double acc0[2] = {0.0, 0.0}, acc1[2] = {0.0, 0.0};  // coarse wedges 0 and 1
    for (int f = 0; f < kFineWedges; ++f) {
        // Y = A_f[di][dj] (rows 6 di.., cols 6 dj..) x P, k = 0..7 in two steps
        double y[2] = {0.0, 0.0};
#pragma unroll
        for (int ks = 0; ks < 2; ++ks) {
            const int    k  = ks * 4 + fr_col;
            const double a  = (fr_row < 6 && k < 6) ? Af[f][6 * bdi + fr_row][6 * bdj + k] : 0.0;
            const double bb = (k < 6 && fr_row < 6) ? P[f][k][fr_row] : 0.0;  // B[k][col = lane >> 2]
            dmma_8x8x4(y, a, bb);
        }
        Yb[b][fr_row][2 * fr_col]     = y[0];
        Yb[b][fr_row][2 * fr_col + 1] = y[1];
        __syncwarp();
        const bool to0 = target_wedge(f >> 1, f & 1) == 0;
#pragma unroll
        for (int ks = 0; ks < 2; ++ks) {
            const int    k  = ks * 4 + fr_col;
            const double a  = (fr_row < 6 && k < 6) ? P[f][k][fr_row] : 0.0;  // (P^T)[row][k]
            const double bb = Yb[b][k][fr_row];                                // Y[k][col = lane >> 2]
            if (to0)
                dmma_8x8x4(acc0, a, bb);
            else
                dmma_8x8x4(acc1, a, bb);
        }
        __syncwarp();  // Yb[b] is rewritten by the next fine wedge
    }
#pragma unroll
    for (int e = 0; e < 2; ++e) {
        const int r = fr_row, c = 2 * fr_col + e;
        if (r >= 6 || c >= 6) continue;
        const int i = 6 * bdi + r, j = 6 * bdj + c;
        if (i > j) continue;
        A.out[static_cast<int64_t>(0 * kPack + pidx(i, j)) * A.nout + slot] = acc0[e];
        A.out[static_cast<int64_t>(1 * kPack + pidx(i, j)) * A.nout + slot] = acc1[e];
    }
}

// Coarse hexes over on-the-fly fine matrices. The fine element matrix is
// A_f[(n,a)][(m,b)] = kwJ (delta_ab g_n.g_m + g_n[b] g_m[a] - 2/3 g_n[a] g_m[b]) (load_fine_matrix), and with
// P_vec = I_3 (x) P the triple product keeps that form with the gradients replaced by h_c = sum_n P[n][c] g_n
// (the coarse shape-function gradients seen from the fine wedge):
// (P^T A_f P)[(c,a)][(e,b)] = kwJ (delta_ab h_c.h_e + h_c[b] h_e[a] - 2/3 h_c[a] h_e[b]).
// Each fine wedge then costs 18 six-term sums and one rank-structured update of the 171 packed entries per
// coarse wedge instead of two 18 x 18 x 6 products; exact in exact arithmetic, rounding differs from the
// triple product in the last bits. The set-up is spread over the CTA in three short phases: the geometry of
// the four fine columns and the 96 rows of the 16 interpolation matrices; the 16 x 18 gradients and the 16
// weights; the 16 x 18 entries of h. Thread (t, p) of the first 342 then sums entry p of coarse wedge t over
// the 8 fine wedges it receives.
constexpr int kRankThreads = 352;

__global__ void __launch_bounds__(kRankThreads, 3) gca_build_rank_kernel(GcaBuildArgs A)
{
    const int nlf = A.nlf, nrf = A.nrf;
    int       slot, d, xc, yc, rc;
    if (!coarse_cell_of_block(A, slot, d, xc, yc, rc)) return;

    __shared__ double Gw[4][20];  // column_geometry of fine column q = x + 2 y (both wedges)
    __shared__ double P[kFineWedges][6][6];
    __shared__ double G[kFineWedges][6][3];
    __shared__ double H[kFineWedges][6][3];
    __shared__ double kw[kFineWedges];

    const int tid = threadIdx.x;
    if (tid < 4) {
        column_geometry<double>(A.coords, nlf, d, 2 * xc + (tid & 1), 2 * yc + (tid >> 1), Gw[tid]);
    } else if (tid >= 32 && tid < 32 + 6 * kFineWedges) {
        const int f = (tid - 32) / 6, fl = (tid - 32) % 6;
        int       fx, fy, fr;
        fine_hex(f >> 1, xc, yc, rc, fx, fy, fr);
        interp_row(d, fx, fy, fr, f & 1, fl, nlf, nrf, A.linw, P[f][fl]);
    }
    __syncthreads();
    if (tid < kFineWedges * 18) {
        // gradient component c of shape function n of fine wedge f (as fine_wedge_factors)
        const int     f = tid / 18, n = (tid % 18) / 3, c = tid % 3, h = f >> 1, w = f & 1;
        const int     fr = 2 * rc + (h >> 2);
        const double  r0 = A.radii[fr], r1 = A.radii[fr + 1];
        const double  rm = 0.5 * (r0 + r1), hdr = 0.5 * (r1 - r0);
        const double  alpha = 0.5 / rm, beta = 1.0 / (6.0 * hdr);
        const double* gw = Gw[h & 3] + 10 * w;
        const int     m  = n % 3;
        const double  sg = n < 3 ? -1.0 : 1.0;
        const double  L  = m == 0 ? -(gw[c] + gw[3 + c]) : (m == 1 ? gw[c] : gw[3 + c]);
        G[f][n][c]       = alpha * L + sg * beta * gw[6 + c];
    } else if (tid >= 288 && tid < 288 + kFineWedges) {
        const int f = tid - 288, h = f >> 1, w = f & 1;
        int       fx, fy, fr;
        fine_hex(h, xc, yc, rc, fx, fy, fr);
        const double r0 = A.radii[fr], r1 = A.radii[fr + 1];
        const double rm = 0.5 * (r0 + r1), hdr = 0.5 * (r1 - r0);
        double       kv;
        if (A.kq0) {
            kv = A.kq0[node_index(nlf - 1, nrf - 1, d, fx, fy, fr)];
        } else {
            const double wlat0 = 1.0 - 1.0 / 3.0 - 1.0 / 3.0, wlat = 1.0 / 3.0;
            kv                 = 0.0;
            for (int n = 0; n < 6; ++n)
                kv += (n % 3 == 0 ? wlat0 : wlat) * 0.5 *
                      A.k[node_index(nlf, nrf, d, fx + woff(w, n, 0), fy + woff(w, n, 1), fr + woff(w, n, 2))];
        }
        kw[f] = kv * Gw[h & 3][10 * w + 9] * rm * rm * hdr;
    }
    __syncthreads();
    if (tid < kFineWedges * 18) {
        const int f = tid / 18, c = (tid % 18) / 3, a = tid % 3;
        double    h = 0.0;
#pragma unroll
        for (int n = 0; n < 6; ++n) h += P[f][n][c] * G[f][n][a];
        H[f][c][a] = h;
    }
    __syncthreads();
    if (tid >= 2 * kPack) return;
    const int t = tid / kPack, p = tid % kPack;
    int       i, j;
    packed_pair(p, i, j);
    const int ni = i % 6, di = i / 6, nj = j % 6, dj = j / 6;
    double    acc = 0.0;
    for (int f = 0; f < kFineWedges; ++f) {
        if (target_wedge(f >> 1, f & 1) != t) continue;
        const double* hi = H[f][ni];
        const double* hj = H[f][nj];
        double        v  = hi[dj] * hj[di] - (2.0 / 3.0) * hi[di] * hj[dj];
        if (di == dj) v += hi[0] * hj[0] + hi[1] * hj[1] + hi[2] * hj[2];
        acc += kw[f] * v;
    }
    A.out[static_cast<int64_t>(t * kPack + p) * A.nout + slot] = acc;
}

// Element matrices of one level itself (no coarsening): the stored form of the
// on-the-fly operator (get_local_matrix of a level without stored matrices).
// Slot s of out holds cell cells[s] (or s); with base given, out = base - A_e
// (the correction of selectively stored matrices over the on-the-fly ones).
__global__ void __launch_bounds__(kN * kN) element_matrices_kernel(GcaBuildArgs A, const double* base)
{
    const int nl = A.nlf, nr = A.nrf;
    const int slot = blockIdx.x;
    if (slot >= A.nout) return;
    int d, x, y, r;
    decode_cell(A.cells ? A.cells[slot] : slot, nl, nr, d, x, y, r);
    const int i = threadIdx.x / kN, j = threadIdx.x % kN;
    __shared__ double Af[kN][kN];
    __shared__ double G[6][3];
    __shared__ double kwJ;
    for (int w = 0; w < 2; ++w) {
        load_fine_matrix(A, d, x, y, r, w, Af, G, kwJ);
        if (i <= j) {
            const int64_t o = static_cast<int64_t>(w * kPack + pidx(i, j)) * A.nout + slot;
            A.out[o]        = base ? base[o] - Af[i][j] : Af[i][j];
        }
        __syncthreads();
    }
}

// full[p][cells[s]] = compact[p][s] for the 342 values of every slot
__global__ void scatter_slots_kernel(int nslots, const int* cells, const double* compact, int ncells, double* full)
{
    const int64_t n = static_cast<int64_t>(2 * kPack) * nslots;
    for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < n;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t p = e / nslots, s = e % nslots;
        full[p * ncells + cells[s]] = compact[e];
    }
}

// GCAElementsCollector (gca_elements_collector.hpp:61-103): the gradient of the nodal coefficient in the
// reference coordinates of each wedge at the one-point rule's point (1/3, 1/3, 0) (grad_shape, integrands.hpp:
// 228-235; quad_felippa_1x1, quadrature.hpp:36-39); where its norm exceeds 10 the coarsest ancestor of the cell
// (level_range halvings of each cell index, map_to_coarse_element) is marked. Terms are summed in the
// reference's order so that the comparison sees the same value.
__global__ void gca_mark_kernel(int nl, int nr, const double* k, int level_range, uint8_t* marks)
{
    const int nlc = ((nl - 1) >> level_range) + 1, nrc = ((nr - 1) >> level_range) + 1;
    const int nc  = 10 * (nl - 1) * (nl - 1) * (nr - 1);
    for (int cell = blockIdx.x * blockDim.x + threadIdx.x; cell < nc; cell += gridDim.x * blockDim.x) {
        int d, x, y, r;
        decode_cell(cell, nl, nr, d, x, y, r);
        bool hit = false;
        for (int w = 0; w < 2; ++w) {
            double g[3] = {0.0, 0.0, 0.0};
            for (int n = 0; n < 6; ++n) {
                const double kn = k[node_index(nl, nr, d, x + woff(w, n, 0), y + woff(w, n, 1), r + woff(w, n, 2))];
                const int    m  = n % 3;
                const double srad = 0.5;                                 // 0.5 (1 -+ zeta) at zeta = 0
                const double gxi  = m == 0 ? -1.0 : (m == 1 ? 1.0 : 0.0);  // grad_shape_lat_xi
                const double geta = m == 0 ? -1.0 : (m == 2 ? 1.0 : 0.0);  // grad_shape_lat_eta
                const double slat = m == 0 ? 1.0 - 1.0 / 3.0 - 1.0 / 3.0 : 1.0 / 3.0;
                const double grad = n < 3 ? -0.5 : 0.5;                  // grad_shape_rad
                // separate roundings (no fused multiply-add), as the reference computes it
                g[0] = __dadd_rn(g[0], __dmul_rn(__dmul_rn(gxi, srad), kn));
                g[1] = __dadd_rn(g[1], __dmul_rn(__dmul_rn(geta, srad), kn));
                g[2] = __dadd_rn(g[2], __dmul_rn(__dmul_rn(slat, grad), kn));
            }
            double sum = 0.0;
            for (int c = 0; c < 3; ++c) sum = __dadd_rn(sum, __dmul_rn(g[c], g[c]));
            if (sqrt(sum) > 10.0) hit = true;
        }
        if (hit)
            marks[node_index(nlc - 1, nrc - 1, d, x >> level_range, y >> level_range, r >> level_range)] = 1;
    }
}

// Bake boundary conditions into the matrices of boundary cells (see header).
struct GcaBakeArgs {
    int           nl, nr;  // coarse level dims
    const double* coords;
    const double* radii;
    int           bc_cmb, bc_surf;
    double*       mats;           // in/out [342][stride]
    const int*    cells = nullptr;  // selective storage: slot s holds cells[s]; nullptr: slot = cell
    int           nslots = 0;       // slots of a selective store
};

__device__ void frame(const double* coords, const double* radii, int nl, int d, int x, int y, int r, double (&R)[3][3])
{
    const double* c = coords + lat_index3(nl, d, x, y) * 3;
    double        n[3] = {c[0] * radii[r], c[1] * radii[r], c[2] * radii[r]};
    const double  m    = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    for (int k = 0; k < 3; ++k) n[k] /= m;
    trafo_nt<double>(n, R);
}

// One CTA of 18 x 18 threads per (boundary cell, wedge); thread (i, j) owns
// matrix entry (i, j).
__global__ void __launch_bounds__(kN * kN) gca_bake_kernel(GcaBakeArgs A)
{
    const int nl = A.nl, nr = A.nr;
    const int w = blockIdx.x & 1;
    int       d, x, y, r, side;
    int64_t   cell, stride;
    if (A.cells) {
        // every stored cell; those off the boundary keep their matrices
        const int slot = blockIdx.x >> 1;
        decode_cell(A.cells[slot], nl, nr, d, x, y, r);
        side   = r == 0 ? 0 : (r == nr - 2 ? 1 : -1);  // CMB first on a one-cell shell, as the slow path
        cell   = slot;
        stride = A.nslots;
        if (side < 0) return;
    } else {
        const int nb  = 10 * (nl - 1) * (nl - 1);
        const int idx = blockIdx.x >> 1;  // boundary cell: 10 (nl-1)^2 per side
        side          = idx / nb;
        int t         = idx % nb;
        y             = t % (nl - 1);
        t /= (nl - 1);
        x      = t % (nl - 1);
        d      = t / (nl - 1);
        r      = side == 0 ? 0 : nr - 2;
        cell   = node_index(nl - 1, nr - 1, d, x, y, r);
        stride = 10 * (nl - 1) * (nl - 1) * (nr - 1);
        if (side == 1 && r == 0) return;  // one radial cell: the slow path treats it as CMB only
    }
    const int bc = side == 0 ? A.bc_cmb : A.bc_surf;
    if (bc != 1 && bc != 2) return;
    const int64_t nc = stride;
    const int     tid  = threadIdx.x;
    const int     i = tid / kN, j = tid % kN;
    const int     n0 = side == 0 ? 0 : 3;  // boundary nodes n0..n0+2 of the wedge

    __shared__ double M[kN][kN];      // dimension-wise ordering (node + 6 comp)
    __shared__ double B[kN][kN];      // node-wise ordering (3 node + comp)
    __shared__ double Rn[6][3][3];    // frames (identity off the boundary)
    M[i][j] = A.mats[static_cast<int64_t>(w * kPack + pidx(i, j)) * nc + cell];
    if (bc == 1) {
        // keep the same-dimension diagonal only (epsilon_divdiv_kerngen.hpp:1087-1112)
        const int  na = i % 6, nbn = j % 6;
        const bool ba = na >= n0 && na < n0 + 3, bb = nbn >= n0 && nbn < n0 + 3;
        if (i <= j) {
            const double v = ((ba || bb) && i != j) ? 0.0 : M[i][j];
            A.mats[static_cast<int64_t>(w * kPack + pidx(i, j)) * nc + cell] = v;
        }
        return;
    }
    // free-slip: R^T (Mask o (R A R^T)) R in node-wise ordering (:1113-1192)
    if (tid < 6) {
        const int n = tid;
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) Rn[n][a][b] = (a == b) ? 1.0 : 0.0;
        if (n >= n0 && n < n0 + 3) frame(A.coords, A.radii, nl, d, x + woff(w, n, 0), y + woff(w, n, 1),
                                         r + (side == 0 ? 0 : 1), Rn[n]);
    }
    __syncthreads();
    {
        const int na = i / 3, ca = i % 3, nbn = j / 3, cb = j % 3;
        double    s = 0.0;
        for (int p = 0; p < 3; ++p)
            for (int q = 0; q < 3; ++q) s += Rn[na][ca][p] * M[na + 6 * p][nbn + 6 * q] * Rn[nbn][cb][q];
        const bool ma = (i % 3 == 0) && na >= n0 && na < n0 + 3;  // normal component of a boundary node
        const bool mb = (j % 3 == 0) && nbn >= n0 && nbn < n0 + 3;
        B[i][j]       = ((ma || mb) && i != j) ? 0.0 : s;
    }
    __syncthreads();
    {
        const int ni = i % 6, ci = i / 6, nj = j % 6, cj = j / 6;
        double    s = 0.0;
        for (int p = 0; p < 3; ++p)
            for (int q = 0; q < 3; ++q) s += Rn[ni][p][ci] * B[ni * 3 + p][nj * 3 + q] * Rn[nj][q][cj];
        M[i][j] = s;
    }
    __syncthreads();
    if (i <= j) A.mats[static_cast<int64_t>(w * kPack + pidx(i, j)) * nc + cell] = 0.5 * (M[i][j] + M[j][i]);
}

// Stored-matrix apply: dst += A src. One thread per (cell, wedge), cells
// fastest so that each packed value is one coalesced load across a warp; on
// large levels the matrix streams through L2 with evict-first loads (it is
// read once per apply) while src / dst stay cached. The 171 packed entries are
// walked in a fully unrolled loop whose (row, column) pairs are compile-time
// constants, keeping the 18 inputs and 18 outputs in registers.
template <typename T>
struct GcaApplyArgs {
    int        nl, nr;
    const T*   mats;  // [342][cells] or, selective, [342][nslots]
    const T*   src[3];
    T*         dst[3];
    const int* cells  = nullptr;  // selective storage: slot s holds cells[s]
    int        nslots = 0;
};

__host__ __device__ constexpr int pair_row(int p)
{
    int a = 0;
    while (p >= kN - a) {
        p -= kN - a;
        ++a;
    }
    return a;
}
__host__ __device__ constexpr int pair_col(int p)
{
    int a = 0;
    while (p >= kN - a) {
        p -= kN - a;
        ++a;
    }
    return a + p;
}

// Matrix loads: evict-first where a level's matrices are too large to stay in
// L2 between applies (they are read once per apply); plain loads where they
// fit, so that the consecutive applies of one smoothing sweep find them in L2
// (the level-4 FP32 matrices of a level-6 hierarchy, 56 MB).
constexpr int64_t kGcaStreamBytes = 64ll << 20;

template <typename T, bool kStream>
__device__ __forceinline__ T ld_mat(const T* p)
{
    if constexpr (kStream)
        return __ldcs(p);
    else
        return __ldg(p);
}

// o += A s over packed entries P.. with compile-time (row, column)
template <typename T, bool kStream, int P>
__device__ __forceinline__ void packed_matvec(const T* m, int64_t nc, const T (&s)[kN], T (&o)[kN])
{
    if constexpr (P < kPack) {
        constexpr int a = pair_row(P), b = pair_col(P);
        const T       v = ld_mat<T, kStream>(m + static_cast<int64_t>(P) * nc);
        if constexpr (a == b) {
            o[a] += v * s[a];
        } else {
            o[a] += v * s[b];
            o[b] += v * s[a];
        }
        packed_matvec<T, kStream, P + 1>(m, nc, s, o);
    }
}

template <typename T, bool kStream>
__global__ void __launch_bounds__(128, 3) gca_apply_kernel(GcaApplyArgs<T> A)
{
    const int nl = A.nl, nr = A.nr;
    const int nc  = A.cells ? A.nslots : 10 * (nl - 1) * (nl - 1) * (nr - 1);
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= 2 * nc) return;
    const int w    = idx >= nc ? 1 : 0;
    const int cell = idx - w * nc;  // slot of the matrix
    int       d, x, y, r;
    decode_cell(A.cells ? A.cells[cell] : cell, nl, nr, d, x, y, r);
    int64_t id[6];
    T         s[kN], o[kN];
#pragma unroll
    for (int n = 0; n < 6; ++n) {
        id[n] = node_index(nl, nr, d, x + woff(w, n, 0), y + woff(w, n, 1), r + woff(w, n, 2));
#pragma unroll
        for (int c = 0; c < 3; ++c) s[n + 6 * c] = A.src[c][id[n]];
    }
#pragma unroll
    for (int a = 0; a < kN; ++a) o[a] = T(0);
    const T* m = A.mats + static_cast<int64_t>(w * kPack) * nc + cell;
    packed_matvec<T, kStream, 0>(m, nc, s, o);
#pragma unroll
    for (int n = 0; n < 6; ++n)
#pragma unroll
        for (int c = 0; c < 3; ++c) atomicAdd(&A.dst[c][id[n]], o[n + 6 * c]);
}

// Diagonal mode of the stored operator applied to src: plain diagonal on
// interior / Dirichlet cells, R^T diag(R A R^T o Mask) R on free-slip cells
// (epsilon_divdiv_kerngen.hpp:1205-1240 with diagonal_ == true). Uses the
// unbaked matrices.
struct GcaDiagArgs {
    int           nl, nr;
    const double* coords;
    const double* radii;
    int           bc_cmb, bc_surf;
    const double* mats;  // unbaked
    const double* src[3];
    double*       dst[3];
    const int*    cells  = nullptr;  // selective storage: slot s holds cells[s]
    int           nslots = 0;
};

// cell (d, x, y, r) whose two wedge matrices start at m (value stride nc)
__device__ void diag_cell(const GcaDiagArgs& A, int d, int x, int y, int r, const double* mbase, int64_t nc)
{
    const int nl = A.nl, nr = A.nr;
    const int side = r == 0 ? 0 : (r == nr - 2 ? 1 : -1);
    const int bc   = side == 0 ? A.bc_cmb : (side == 1 ? A.bc_surf : 0);
    for (int w = 0; w < 2; ++w) {
        int64_t id[6];
        for (int n = 0; n < 6; ++n) id[n] = node_index(nl, nr, d, x + woff(w, n, 0), y + woff(w, n, 1), r + woff(w, n, 2));
        const double* m = mbase + static_cast<int64_t>(w * kPack) * nc;
        const int     n0 = side == 0 ? 0 : 3;
        for (int n = 0; n < 6; ++n) {
            const bool bnode = (bc == 2) && n >= n0 && n < n0 + 3;
            double     out[3];
            if (!bnode) {
                for (int c = 0; c < 3; ++c) out[c] = m[static_cast<int64_t>(pidx(n + 6 * c, n + 6 * c)) * nc] * A.src[c][id[n]];
            } else {
                double R[3][3];
                frame(A.coords, A.radii, nl, d, x + woff(w, n, 0), y + woff(w, n, 1), r + side, R);
                double Ab[3][3];
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b) Ab[a][b] = m[static_cast<int64_t>(pidx(n + 6 * a, n + 6 * b)) * nc];
                double sv[3] = {A.src[0][id[n]], A.src[1][id[n]], A.src[2][id[n]]}, v[3];
                for (int a = 0; a < 3; ++a) {
                    double dg = 0.0;  // (R Ab R^T)_{aa}
                    for (int p = 0; p < 3; ++p)
                        for (int q = 0; q < 3; ++q) dg += R[a][p] * Ab[p][q] * R[a][q];
                    const double rs = R[a][0] * sv[0] + R[a][1] * sv[1] + R[a][2] * sv[2];
                    v[a]            = dg * rs;
                }
                for (int c = 0; c < 3; ++c) out[c] = R[0][c] * v[0] + R[1][c] * v[1] + R[2][c] * v[2];
            }
            for (int c = 0; c < 3; ++c) atomicAdd(&A.dst[c][id[n]], out[c]);
        }
    }
}

__global__ void gca_diag_kernel(GcaDiagArgs A)
{
    const int nl = A.nl, nr = A.nr;
    const int nc = 10 * (nl - 1) * (nl - 1) * (nr - 1);
    const int r  = blockIdx.x * blockDim.x + threadIdx.x;
    const int y  = blockIdx.y % (nl - 1), x = blockIdx.y / (nl - 1), d = blockIdx.z;
    if (r >= nr - 1) return;
    const int64_t cell = node_index(nl - 1, nr - 1, d, x, y, r);
    diag_cell(A, d, x, y, r, A.mats + cell, nc);
}

// the same over the slots of a selective store
__global__ void gca_diag_slots_kernel(GcaDiagArgs A)
{
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= A.nslots) return;
    int d, x, y, r;
    decode_cell(A.cells[slot], A.nl, A.nr, d, x, y, r);
    diag_cell(A, d, x, y, r, A.mats + slot, A.nslots);
}

__global__ void f64_to_f32(int64_t n, const double* in, float* out)
{
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        out[i] = static_cast<float>(in[i]);
}

inline int launch_status(int kernels = 1)
{
    note_launch(kernels);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}
inline dim3 cell_grid(int nl, int nr, int thr) { return dim3((nr - 1 + thr - 1) / thr, (nl - 1) * (nl - 1), 10); }

}  // namespace

int gca_values_per_cell() { return 2 * kPack; }

namespace {
constexpr int kMaxDevices = 64;  // devices a process can drive

// the mma build's dynamic shared-memory limit, raised once per device
int mma_smem_configure()
{
    static std::mutex mu;
    static bool       done[kMaxDevices] = {};
    int               dev               = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return -1;
    std::lock_guard<std::mutex> lock(mu);
    if (!done[dev]) {
        if (cudaFuncSetAttribute(gca_build_mma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(kMmaSmem)) != cudaSuccess)
            return -1;
        done[dev] = true;
    }
    return 0;
}
}  // namespace

int gca_build(int nlf, int nrf, const double* coords_f, const double* radii_f, const double* k_f, const double* kq0_f,
              const double* fine_mats, double* coarse_mats, cudaStream_t st, const double* linear_weights,
              bool tensor_cores, const GcaSlots& sl)
{
    GcaBuildArgs a;
    a.nlf       = nlf;
    a.nrf       = nrf;
    a.coords    = coords_f;
    a.radii     = radii_f;
    a.k         = k_f;
    a.kq0       = kq0_f;
    a.fine_mats = fine_mats;
    a.out       = coarse_mats;
    a.linw      = linear_weights;
    const int nlc = (nlf + 1) / 2, nrc = (nrf + 1) / 2;
    const int ncc = 10 * (nlc - 1) * (nlc - 1) * (nrc - 1);
    a.cells       = sl.cells;
    a.nout        = sl.cells ? sl.nslots : ncc;
    a.fine_slot   = sl.fine_slot;
    a.fine_stride = sl.fine_slot ? sl.fine_stride : 10 * (nlf - 1) * (nlf - 1) * (nrf - 1);
    a.err         = sl.err;
    if (a.nout == 0) return 0;
    if (!tensor_cores) {
        gca_build_kernel<<<a.nout, kN * kN, 0, st>>>(a);
    } else if (fine_mats == nullptr) {
        gca_build_rank_kernel<<<a.nout, kRankThreads, 0, st>>>(a);
    } else {
        if (mma_smem_configure() != 0) return -1;
        gca_build_mma_kernel<<<a.nout, kMmaThreads, kMmaSmem, st>>>(a);
    }
    return launch_status();
}

int element_matrices(int nl, int nr, const double* coords, const double* radii, const double* k, const double* kq0,
                     double* mats, cudaStream_t st, const int* cells, int nslots, const double* base)
{
    GcaBuildArgs a;
    a.nlf    = nl;
    a.nrf    = nr;
    a.coords = coords;
    a.radii  = radii;
    a.k      = k;
    a.kq0    = kq0;
    a.out    = mats;
    a.cells  = cells;
    a.nout   = cells ? nslots : 10 * (nl - 1) * (nl - 1) * (nr - 1);
    if (a.nout == 0) return 0;
    element_matrices_kernel<<<a.nout, kN * kN, 0, st>>>(a, base);
    return launch_status();
}

int gca_scatter_slots(int nslots, const int* cells, const double* compact, int ncells, double* full, cudaStream_t st)
{
    if (nslots == 0) return 0;
    scatter_slots_kernel<<<1184, 256, 0, st>>>(nslots, cells, compact, ncells, full);
    return launch_status();
}

int gca_mark_elements(int nl, int nr, const double* k, int level_range, uint8_t* marks, cudaStream_t st)
{
    const int nc = 10 * (nl - 1) * (nl - 1) * (nr - 1);
    gca_mark_kernel<<<(nc + 255) / 256, 256, 0, st>>>(nl, nr, k, level_range, marks);
    return launch_status();
}

int gca_bake_boundary(int nl, int nr, const double* coords, const double* radii, int bc_cmb, int bc_surf, double* mats,
                      cudaStream_t st, const int* cells, int nslots)
{
    GcaBakeArgs a{nl, nr, coords, radii, bc_cmb, bc_surf, mats, cells, nslots};
    if ((bc_cmb != 1 && bc_cmb != 2) && (bc_surf != 1 && bc_surf != 2)) return 0;
    const int n = cells ? nslots : 2 * 10 * (nl - 1) * (nl - 1);  // stored cells, or boundary cells of both sides
    if (n == 0) return 0;
    gca_bake_kernel<<<2 * n, kN * kN, 0, st>>>(a);
    return launch_status();
}

template <typename T>
int gca_apply_add(int nl, int nr, const T* mats, const T* const* src, T* const* dst, cudaStream_t st,
                  const int* cells, int nslots)
{
    GcaApplyArgs<T> a{};
    a.nl   = nl;
    a.nr   = nr;
    a.mats = mats;
    for (int c = 0; c < 3; ++c) {
        a.src[c] = src[c];
        a.dst[c] = dst[c];
    }
    a.cells         = cells;
    a.nslots        = nslots;
    const int items = 2 * (cells ? nslots : 10 * (nl - 1) * (nl - 1) * (nr - 1));
    if (items == 0) return 0;
    const bool stream = static_cast<int64_t>(items) * kPack * static_cast<int64_t>(sizeof(T)) > kGcaStreamBytes;
    const int  blocks = (items + 127) / 128;
    if (stream)
        gca_apply_kernel<T, true><<<blocks, 128, 0, st>>>(a);
    else
        gca_apply_kernel<T, false><<<blocks, 128, 0, st>>>(a);
    return launch_status();
}
template int gca_apply_add<double>(int, int, const double*, const double* const*, double* const*, cudaStream_t,
                                   const int*, int);
template int gca_apply_add<float>(int, int, const float*, const float* const*, float* const*, cudaStream_t,
                                  const int*, int);

int gca_diag_add(int nl, int nr, const double* coords, const double* radii, int bc_cmb, int bc_surf,
                 const double* mats, const double* const* src, double* const* dst, cudaStream_t st, const int* cells,
                 int nslots)
{
    GcaDiagArgs a{};
    a.nl = nl;
    a.nr = nr;
    a.coords = coords;
    a.radii  = radii;
    a.bc_cmb = bc_cmb;
    a.bc_surf = bc_surf;
    a.mats    = mats;
    for (int c = 0; c < 3; ++c) {
        a.src[c] = src[c];
        a.dst[c] = dst[c];
    }
    if (cells) {
        a.cells  = cells;
        a.nslots = nslots;
        if (nslots == 0) return 0;
        gca_diag_slots_kernel<<<(nslots + 127) / 128, 128, 0, st>>>(a);
        return launch_status();
    }
    const int thr = nr - 1 >= 64 ? 64 : 32;
    gca_diag_kernel<<<cell_grid(nl, nr, thr), thr, 0, st>>>(a);
    return launch_status();
}

int gca_to_f32(int64_t n, const double* in, float* out, cudaStream_t st)
{
    f64_to_f32<<<1184, 256, 0, st>>>(n, in, out);
    return launch_status();
}

}  // namespace tn
