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

// Interpolation matrix P[fine node][coarse node] of fine wedge (fx, fy, fr, w)
// (gca.hpp:204-383): InterpolationMode::Constant, or InterpolationMode::Linear when linw (the fine level's
// linear-transfer weights, two per node: prolongation_linear_weights) is given.
__device__ void interp_matrix(int d, int fx, int fy, int fr, int w, int nlf, int nrf, const double* linw,
                              double (&P)[6][6])
{
    for (int a = 0; a < 6; ++a)
        for (int b = 0; b < 6; ++b) P[a][b] = 0.0;
    for (int fl = 0; fl < 6; ++fl) {
        const int ix = fx + woff(w, fl, 0), iy = fy + woff(w, fl, 1), ir = fr + woff(w, fl, 2);
        if (ix % 2 == 0 && iy % 2 == 0 && ir % 2 == 0) {
            P[fl][fl] = 1.0;
            continue;
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
            P[fl][a]     = linw ? lw0 : 0.5;
            P[fl][a + 3] = linw ? lw1 : 0.5;
            continue;
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
            P[fl][c0] = lw0;
            P[fl][c1] = lw0;
            P[fl][c2] = lw1;
            P[fl][c3] = lw1;
            continue;
        }
        P[fl][c0] = pweight(ix, iy, ir, x0, y0, rb);
        P[fl][c1] = pweight(ix, iy, ir, x1, y1, rb);
        P[fl][c2] = pweight(ix, iy, ir, x0, y0, rt);
        P[fl][c3] = pweight(ix, iy, ir, x1, y1, rt);
    }
}

// coarse wedge receiving fine hex h (x + 2 y + 4 r shift order of gca.hpp:176-185) wedge w
__host__ __device__ __forceinline__ int target_wedge(int h, int w)
{
    const int hl = h & 3;  // lateral position in the coarse hex: 0 (0,0) 1 (1,0) 2 (0,1) 3 (1,1)
    if (w == 0) return hl == 3 ? 1 : 0;
    return hl == 0 ? 0 : 1;
}

struct GcaBuildArgs {
    int           nlf, nrf;       // fine level dims
    const double* coords;         // fine coords
    const double* radii;          // fine radii
    const double* k;              // fine nodal coefficient (on-the-fly matrices) or nullptr
    const double* kq0;            // fine cell coefficient or nullptr
    const double* fine_mats;      // stored fine matrices [342][fine cells] or nullptr
    double*       out;            // coarse matrices [342][coarse cells]
    const double* linw = nullptr; // fine linear-transfer weights (linear interpolation) or nullptr (constant)
};

// Fine wedge matrix of (d, fx, fy, fr, w) into Af (dimension-wise ordering),
// either assembled on the fly or read from stored matrices. Called by all
// 18 x 18 threads of the CTA; ends with the matrix visible to all of them.
__device__ void load_fine_matrix(const GcaBuildArgs& A, int d, int fx, int fy, int fr, int w, double (&Af)[kN][kN],
                                 double (&G)[6][3], double& kwJ)
{
    const int  nlf = A.nlf, nrf = A.nrf;
    const int  tid = threadIdx.x;
    const bool ent = tid < kN * kN;  // threads beyond the 324 entries only take part in the barrier
    const int  i = ent ? tid / kN : 0, j = ent ? tid % kN : 0;
    const int  ni = i % 6, di = i / 6, nj = j % 6, dj = j / 6;
    if (A.fine_mats == nullptr) {
        // element matrix: gradients and k|det J| first
        if (tid == 0) {
            double geo[20];
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
        __syncthreads();
        // A(i,j) = kwJ [delta_{di dj} g_i.g_j + g_i[dj] g_j[di] - 2/3 g_i[di] g_j[dj]]
        const double gij = (di == dj) ? (G[ni][0] * G[nj][0] + G[ni][1] * G[nj][1] + G[ni][2] * G[nj][2]) : 0.0;
        if (ent) Af[i][j] = kwJ * (gij + G[ni][dj] * G[nj][di] - (2.0 / 3.0) * G[ni][di] * G[nj][dj]);
    } else if (ent) {
        const int     ncf = 10 * (nlf - 1) * (nlf - 1) * (nrf - 1);
        const int64_t fc  = node_index(nlf - 1, nrf - 1, d, fx, fy, fr);
        Af[i][j]          = A.fine_mats[static_cast<int64_t>(w * kPack + pidx(i, j)) * ncf + fc];
    }
}

__global__ void __launch_bounds__(kN * kN) gca_build_kernel(GcaBuildArgs A)
{
    const int nlf = A.nlf, nrf = A.nrf;
    const int nlc = (nlf + 1) / 2, nrc = (nrf + 1) / 2;
    const int ncc = 10 * (nlc - 1) * (nlc - 1) * (nrc - 1);
    const int cell = blockIdx.x;
    if (cell >= ncc) return;
    const int rc = cell % (nrc - 1);
    int       t  = cell / (nrc - 1);
    const int yc = t % (nlc - 1);
    t /= (nlc - 1);
    const int xc = t % (nlc - 1);
    const int d  = t / (nlc - 1);

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
        const int fx = 2 * xc + (h & 1), fy = 2 * yc + ((h >> 1) & 1), fr = 2 * rc + ((h >> 2) & 1);
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
        A.out[static_cast<int64_t>(0 * kPack + pidx(i, j)) * ncc + cell] = acc0;
        A.out[static_cast<int64_t>(1 * kPack + pidx(i, j)) * ncc + cell] = acc1;
    }
}

// The same triple products on the FP64 tensor cores (mma.sync m8n8k4, f64 in and out). P_vec = I_3 (x) P
// couples equal dimensions only, so A_c += P_vec^T A_f P_vec splits into nine 6 x 6 blocks
// A_c[di][dj] += P^T A_f[di][dj] P. Warp b of the first nine owns block b = (di, dj) for both coarse wedges
// and keeps it in two 8 x 8 accumulator fragments (the 6 x 6 blocks and P zero-padded to 8 x 8); per fine
// wedge it runs Y = A_f[di][dj] P (two k = 4 steps) and A_c += P^T Y (two more), staging Y through shared
// memory to turn the accumulator layout into the B-operand layout. The 324 threads of the first eleven warps
// assemble the fine element matrix as in gca_build_kernel.
constexpr int kMmaWarps   = 11;  // 352 threads: 324 matrix entries, warps 0-8 for the nine blocks
constexpr int kMmaThreads = 32 * kMmaWarps;

__device__ __forceinline__ void dmma_8x8x4(double (&d)[2], double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(kMmaThreads) gca_build_mma_kernel(GcaBuildArgs A)
{
    const int nlf = A.nlf, nrf = A.nrf;
    const int nlc = (nlf + 1) / 2, nrc = (nrf + 1) / 2;
    const int ncc  = 10 * (nlc - 1) * (nlc - 1) * (nrc - 1);
    const int cell = blockIdx.x;
    if (cell >= ncc) return;
    const int rc = cell % (nrc - 1);
    int       t  = cell / (nrc - 1);
    const int yc = t % (nlc - 1);
    t /= (nlc - 1);
    const int xc = t % (nlc - 1);
    const int d  = t / (nlc - 1);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int b = warp < 9 ? warp : 0, bdi = b / 3, bdj = b % 3;  // block (di, dj) of this warp
    const int fr_row = lane >> 2, fr_col = lane & 3;             // fragment coordinates (PTX m8n8k4 f64)

    __shared__ double Af[kN][kN];
    __shared__ double P[6][6];
    __shared__ double G[6][3];
    __shared__ double kwJ;
    __shared__ double Yb[9][8][8];

    double acc0[2] = {0.0, 0.0}, acc1[2] = {0.0, 0.0};  // coarse wedges 0 and 1
    for (int h = 0; h < 8; ++h) {
        const int fx = 2 * xc + (h & 1), fy = 2 * yc + ((h >> 1) & 1), fr = 2 * rc + ((h >> 2) & 1);
        for (int w = 0; w < 2; ++w) {
            load_fine_matrix(A, d, fx, fy, fr, w, Af, G, kwJ);
            if (tid == 0) interp_matrix(d, fx, fy, fr, w, nlf, nrf, A.linw, P);
            __syncthreads();
            if (warp < 9) {
                // Y = A_f[di][dj] (rows 6 di.., cols 6 dj..) x P, k = 0..7 in two steps
                double y[2] = {0.0, 0.0};
#pragma unroll
                for (int ks = 0; ks < 2; ++ks) {
                    const int k  = ks * 4 + fr_col;
                    const double a  = (fr_row < 6 && k < 6) ? Af[6 * bdi + fr_row][6 * bdj + k] : 0.0;
                    const double bb = (k < 6 && fr_row < 6) ? P[k][fr_row] : 0.0;  // B[k][col = lane >> 2]
                    dmma_8x8x4(y, a, bb);
                }
                Yb[b][fr_row][2 * fr_col]     = y[0];
                Yb[b][fr_row][2 * fr_col + 1] = y[1];
                __syncwarp();
                const bool to0 = target_wedge(h, w) == 0;
#pragma unroll
                for (int ks = 0; ks < 2; ++ks) {
                    const int    k  = ks * 4 + fr_col;
                    const double a  = (fr_row < 6 && k < 6) ? P[k][fr_row] : 0.0;  // (P^T)[row][k]
                    const double bb = Yb[b][k][fr_row];                          // Y[k][col = lane >> 2]
                    if (to0)
                        dmma_8x8x4(acc0, a, bb);
                    else
                        dmma_8x8x4(acc1, a, bb);
                }
            }
            __syncthreads();
        }
    }
    if (warp < 9) {
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const int r = fr_row, c = 2 * fr_col + e;
            if (r >= 6 || c >= 6) continue;
            const int i = 6 * bdi + r, j = 6 * bdj + c;
            if (i > j) continue;
            A.out[static_cast<int64_t>(0 * kPack + pidx(i, j)) * ncc + cell] = acc0[e];
            A.out[static_cast<int64_t>(1 * kPack + pidx(i, j)) * ncc + cell] = acc1[e];
        }
    }
}

// Element matrices of one level itself (no coarsening): the stored form of the
// on-the-fly operator (get_local_matrix of a level without stored matrices).
__global__ void __launch_bounds__(kN * kN) element_matrices_kernel(GcaBuildArgs A)
{
    const int nl = A.nlf, nr = A.nrf;
    const int nc = 10 * (nl - 1) * (nl - 1) * (nr - 1);
    const int cell = blockIdx.x;
    if (cell >= nc) return;
    const int r = cell % (nr - 1);
    int       t = cell / (nr - 1);
    const int y = t % (nl - 1);
    t /= (nl - 1);
    const int x = t % (nl - 1);
    const int d = t / (nl - 1);
    const int i = threadIdx.x / kN, j = threadIdx.x % kN;
    __shared__ double Af[kN][kN];
    __shared__ double G[6][3];
    __shared__ double kwJ;
    for (int w = 0; w < 2; ++w) {
        load_fine_matrix(A, d, x, y, r, w, Af, G, kwJ);
        if (i <= j) A.out[static_cast<int64_t>(w * kPack + pidx(i, j)) * nc + cell] = Af[i][j];
        __syncthreads();
    }
}

// Bake boundary conditions into the matrices of boundary cells (see header).
struct GcaBakeArgs {
    int           nl, nr;  // coarse level dims
    const double* coords;
    const double* radii;
    int           bc_cmb, bc_surf;
    double*       mats;  // in/out [342][cells]
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
    const int nc = 10 * (nl - 1) * (nl - 1) * (nr - 1);
    const int nb = 10 * (nl - 1) * (nl - 1);
    const int w    = blockIdx.x & 1;
    const int idx  = blockIdx.x >> 1;  // boundary cell: 10 (nl-1)^2 per side
    const int side = idx / nb;
    int       t    = idx % nb;
    const int y = t % (nl - 1);
    t /= (nl - 1);
    const int x  = t % (nl - 1);
    const int d  = t / (nl - 1);
    const int r  = side == 0 ? 0 : nr - 2;
    const int bc = side == 0 ? A.bc_cmb : A.bc_surf;
    if (bc != 1 && bc != 2) return;
    const int64_t cell = node_index(nl - 1, nr - 1, d, x, y, r);
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
// fastest so that each packed value is one coalesced load across a warp; the
// matrix streams through L2 with evict-first loads (it is read once per apply)
// while src / dst stay cached. The 171 packed entries are walked in a fully
// unrolled loop whose (row, column) pairs are compile-time constants, keeping
// the 18 inputs and 18 outputs in registers.
template <typename T>
struct GcaApplyArgs {
    int      nl, nr;
    const T* mats;  // [342][cells]
    const T* src[3];
    T*       dst[3];
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

template <typename T>
__device__ __forceinline__ T ld_stream(const T* p)
{
    return __ldcs(p);
}

// o += A s over packed entries P.. with compile-time (row, column)
template <typename T, int P>
__device__ __forceinline__ void packed_matvec(const T* m, int64_t nc, const T (&s)[kN], T (&o)[kN])
{
    if constexpr (P < kPack) {
        constexpr int a = pair_row(P), b = pair_col(P);
        const T       v = ld_stream(m + static_cast<int64_t>(P) * nc);
        if constexpr (a == b) {
            o[a] += v * s[a];
        } else {
            o[a] += v * s[b];
            o[b] += v * s[a];
        }
        packed_matvec<T, P + 1>(m, nc, s, o);
    }
}

template <typename T>
__global__ void __launch_bounds__(128) gca_apply_kernel(GcaApplyArgs<T> A)
{
    const int nl = A.nl, nr = A.nr;
    const int nc  = 10 * (nl - 1) * (nl - 1) * (nr - 1);
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= 2 * nc) return;
    const int w    = idx >= nc ? 1 : 0;
    const int cell = idx - w * nc;
    const int r    = cell % (nr - 1);
    int       t    = cell / (nr - 1);
    const int y    = t % (nl - 1);
    t /= (nl - 1);
    const int x = t % (nl - 1);
    const int d = t / (nl - 1);
    int64_t   id[6];
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
    packed_matvec<T, 0>(m, nc, s, o);
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
};

__global__ void gca_diag_kernel(GcaDiagArgs A)
{
    const int nl = A.nl, nr = A.nr;
    const int nc = 10 * (nl - 1) * (nl - 1) * (nr - 1);
    const int r  = blockIdx.x * blockDim.x + threadIdx.x;
    const int y  = blockIdx.y % (nl - 1), x = blockIdx.y / (nl - 1), d = blockIdx.z;
    if (r >= nr - 1) return;
    const int64_t cell = node_index(nl - 1, nr - 1, d, x, y, r);
    const int     side = r == 0 ? 0 : (r == nr - 2 ? 1 : -1);
    const int     bc   = side == 0 ? A.bc_cmb : (side == 1 ? A.bc_surf : 0);
    for (int w = 0; w < 2; ++w) {
        int64_t id[6];
        for (int n = 0; n < 6; ++n) id[n] = node_index(nl, nr, d, x + woff(w, n, 0), y + woff(w, n, 1), r + woff(w, n, 2));
        const double* m = A.mats + static_cast<int64_t>(w * kPack) * nc + cell;
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

int gca_build(int nlf, int nrf, const double* coords_f, const double* radii_f, const double* k_f, const double* kq0_f,
              const double* fine_mats, double* coarse_mats, cudaStream_t st, const double* linear_weights,
              bool tensor_cores)
{
    GcaBuildArgs a{nlf, nrf, coords_f, radii_f, k_f, kq0_f, fine_mats, coarse_mats, linear_weights};
    const int    nlc = (nlf + 1) / 2, nrc = (nrf + 1) / 2;
    const int    ncc = 10 * (nlc - 1) * (nlc - 1) * (nrc - 1);
    if (tensor_cores)
        gca_build_mma_kernel<<<ncc, kMmaThreads, 0, st>>>(a);
    else
        gca_build_kernel<<<ncc, kN * kN, 0, st>>>(a);
    return launch_status();
}

int element_matrices(int nl, int nr, const double* coords, const double* radii, const double* k, const double* kq0,
                     double* mats, cudaStream_t st)
{
    GcaBuildArgs a{nl, nr, coords, radii, k, kq0, nullptr, mats};
    element_matrices_kernel<<<10 * (nl - 1) * (nl - 1) * (nr - 1), kN * kN, 0, st>>>(a);
    return launch_status();
}

int gca_bake_boundary(int nl, int nr, const double* coords, const double* radii, int bc_cmb, int bc_surf, double* mats,
                      cudaStream_t st)
{
    GcaBakeArgs a{nl, nr, coords, radii, bc_cmb, bc_surf, mats};
    if ((bc_cmb != 1 && bc_cmb != 2) && (bc_surf != 1 && bc_surf != 2)) return 0;
    const int n = 2 * 10 * (nl - 1) * (nl - 1);  // boundary cells of both sides
    gca_bake_kernel<<<2 * n, kN * kN, 0, st>>>(a);
    return launch_status();
}

template <typename T>
int gca_apply_add(int nl, int nr, const T* mats, const T* const* src, T* const* dst, cudaStream_t st)
{
    GcaApplyArgs<T> a{};
    a.nl   = nl;
    a.nr   = nr;
    a.mats = mats;
    for (int c = 0; c < 3; ++c) {
        a.src[c] = src[c];
        a.dst[c] = dst[c];
    }
    const int items = 2 * 10 * (nl - 1) * (nl - 1) * (nr - 1);
    gca_apply_kernel<T><<<(items + 127) / 128, 128, 0, st>>>(a);
    return launch_status();
}
template int gca_apply_add<double>(int, int, const double*, const double* const*, double* const*, cudaStream_t);
template int gca_apply_add<float>(int, int, const float*, const float* const*, float* const*, cudaStream_t);

int gca_diag_add(int nl, int nr, const double* coords, const double* radii, int bc_cmb, int bc_surf,
                 const double* mats, const double* const* src, double* const* dst, cudaStream_t st)
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
