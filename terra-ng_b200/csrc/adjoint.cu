// Backward (vector-Jacobian product) of the epsilon-div-div apply with respect
// to a per-cell (Q0) log-viscosity: the operator is linear in eta_cell, so
//   d(lambda^T A u) / d log(eta_cell) = lambda_e^T A_e(eta_cell) u_e,
// the cell's own contribution to the bilinear form with the operator's
// boundary treatment (Dirichlet masks, free-slip projection and normal
// stiffness). One thread per cell; the cell math is the one the matrix-free
// kernel uses (tn_wedge_math.cuh), accumulated and reduced in the working
// precision T. The velocity part of the backward pass, A^T lambda = A lambda,
// is the forward apply itself (A is symmetric).
#include "tn_device.cuh"
#include "tn_kernels.hpp"
#include "tn_wedge_math.cuh"

namespace tn {
namespace {

template <typename T>
__global__ void __launch_bounds__(128) vjp_logeta_kernel(VjpLaunch<T> A)
{
    const int nl = A.nl, nr = A.nr;
    const int nc   = 10 * (nl - 1) * (nl - 1) * (nr - 1);
    const int cell = blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= nc) return;
    const int r = cell % (nr - 1);
    int       t = cell / (nr - 1);
    const int y = t % (nl - 1);
    t /= (nl - 1);
    const int x = t % (nl - 1);
    const int d = t / (nl - 1);

    T geo[20];
    column_geometry<T>(A.coords, nl, d, x, y, geo);
    const T r0 = A.radii[r], r1 = A.radii[r + 1];
    const T rm = T(0.5) * (r0 + r1), hdr = T(0.5) * (r1 - r0);
    const T alpha = T(0.5) / rm, beta = T(1) / (T(6) * hdr);
    const T dfac  = rm * rm * hdr;  // Q0: the cell value multiplies the wedge volume directly

    T   u[4][2][3], lam[4][2][3], out[4][2][3], nrm[4][3], ks[4];
    int bcs[2] = {r == 0 ? A.bc_cmb : 0, r + 1 == nr - 1 ? A.bc_surf : 0};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int qx = x + (q & 1), qy = y + (q >> 1);
        const T*  c  = A.coords + lat_index3(nl, d, qx, qy) * 3;
        const T   m  = sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
#pragma unroll
        for (int k = 0; k < 3; ++k) nrm[q][k] = c[k] / m;
        ks[q] = T(0);
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            const int64_t id = node_index(nl, nr, d, qx, qy, r + s);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                u[q][s][k]   = A.u[k][id];
                lam[q][s][k] = A.lam[k][id];
                out[q][s][k] = T(0);
            }
        }
    }
    const T kcell = A.kq0[cell];
    cell_apply<T, false>(u, ks, kcell, true, geo, alpha, beta, dfac, bcs, nrm, out);
    T acc = T(0);
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int s = 0; s < 2; ++s)
#pragma unroll
            for (int k = 0; k < 3; ++k) acc += lam[q][s][k] * out[q][s][k];
    A.grad[cell] = A.accumulate ? A.grad[cell] + acc : acc;
}

inline int launch_status(int kernels = 1)
{
    note_launch(kernels);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

}  // namespace

template <typename T>
int epsdivdiv_vjp_logeta(const VjpLaunch<T>& p, cudaStream_t st)
{
    if (!p.kq0) return -1;
    const int nc = 10 * (p.nl - 1) * (p.nl - 1) * (p.nr - 1);
    vjp_logeta_kernel<T><<<(nc + 127) / 128, 128, 0, st>>>(p);
    return launch_status();
}
template int epsdivdiv_vjp_logeta<double>(const VjpLaunch<double>&, cudaStream_t);
template int epsdivdiv_vjp_logeta<float>(const VjpLaunch<float>&, cudaStream_t);

}  // namespace tn
