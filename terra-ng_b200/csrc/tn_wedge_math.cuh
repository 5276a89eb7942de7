// Per-cell wedge math of the epsilon-div-div operator, shared by the CUDA
// kernels and host-side unit checks (__host__ __device__).
#pragma once

#include <cmath>
#include <cstdint>

namespace tn {

#ifndef TN_NODE_INDEX_DEFINED
#define TN_NODE_INDEX_DEFINED
__host__ __device__ __forceinline__ int64_t lat_index3(int nl, int d, int x, int y)
{
    return (static_cast<int64_t>(d) * nl + x) * nl + y;
}
#endif

// Wedge corner map m -> hex corner q, q = dx + 2 dy (kernel_helpers.hpp:291-312).
__host__ __device__ constexpr int wedge_corner(int w, int m) { return w == 0 ? m : 3 - m; }

template <typename T>
__host__ __device__ __forceinline__ T tabs(T v)
{
    return v < T(0) ? -v : v;
}

// Lateral geometry of one hex column: for each wedge e1, e2, e3 (columns of
// M^{-T}) and det(M). M columns: a1 = p1 - p0, a2 = p2 - p0, a3 = (p0+p1+p2)/3.
template <typename T>
__host__ __device__ void column_geometry(const T* coords, int nl, int d, int x, int y, T* g /*20*/)
{
    T p[4][3];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const T* c = coords + (lat_index3(nl, d, x + (q & 1), y + (q >> 1))) * 3;
        p[q][0]    = c[0];
        p[q][1]    = c[1];
        p[q][2]    = c[2];
    }
#pragma unroll
    for (int w = 0; w < 2; ++w) {
        const T* p0 = p[wedge_corner(w, 0)];
        const T* p1 = p[wedge_corner(w, 1)];
        const T* p2 = p[wedge_corner(w, 2)];
        T        a1[3], a2[3], a3[3];
        for (int i = 0; i < 3; ++i) {
            a1[i] = p1[i] - p0[i];
            a2[i] = p2[i] - p0[i];
            a3[i] = (p0[i] + p1[i] + p2[i]) * (T(1) / T(3));
        }
        // rows of M^{-1}: (a2 x a3, a3 x a1, a1 x a2) / det
        T c23[3] = {a2[1] * a3[2] - a2[2] * a3[1], a2[2] * a3[0] - a2[0] * a3[2], a2[0] * a3[1] - a2[1] * a3[0]};
        T c31[3] = {a3[1] * a1[2] - a3[2] * a1[1], a3[2] * a1[0] - a3[0] * a1[2], a3[0] * a1[1] - a3[1] * a1[0]};
        T c12[3] = {a1[1] * a2[2] - a1[2] * a2[1], a1[2] * a2[0] - a1[0] * a2[2], a1[0] * a2[1] - a1[1] * a2[0]};
        T det    = a1[0] * c23[0] + a1[1] * c23[1] + a1[2] * c23[2];
        T id     = T(1) / det;
        T* o     = g + 10 * w;
        for (int i = 0; i < 3; ++i) {
            o[i]     = c23[i] * id;
            o[3 + i] = c31[i] * id;
            o[6 + i] = c12[i] * id;
        }
        o[9] = det < T(0) ? -det : det;
    }
}

// Normal-tangential frame rows (n, t1, t2) of a unit normal
// (local_basis_trafo_normal_tangential.hpp:34-76).
template <typename T>
__host__ __device__ void trafo_nt(const T n[3], T R[3][3])
{
    T ax = tabs(n[0]), ay = tabs(n[1]), az = tabs(n[2]);
    T ref[3] = {0, 0, 0};
    if (ax <= ay && ax <= az)
        ref[0] = 1;
    else if (ay <= ax && ay <= az)
        ref[1] = 1;
    else
        ref[2] = 1;
    T t1[3] = {ref[1] * n[2] - ref[2] * n[1], ref[2] * n[0] - ref[0] * n[2], ref[0] * n[1] - ref[1] * n[0]};
    T m     = sqrt(t1[0] * t1[0] + t1[1] * t1[1] + t1[2] * t1[2]);
    for (int i = 0; i < 3; ++i) t1[i] /= m;
    T t2[3] = {n[1] * t1[2] - n[2] * t1[1], n[2] * t1[0] - n[0] * t1[2], n[0] * t1[1] - n[1] * t1[0]};
    m       = sqrt(t2[0] * t2[0] + t2[1] * t2[1] + t2[2] * t2[2]);
    for (int i = 0; i < 3; ++i) {
        t2[i] /= m;
        R[0][i] = n[i];
        R[1][i] = t1[i];
        R[2][i] = t2[i];
    }
}

// One hex cell (two wedges). u[q][s][c]: corner q, side s (0 bottom, 1 top).
// ks[q]: k_bot + k_top (nodal) ; kcell used when Q0. Accumulates into out.
// bcs[s]: boundary condition of side s of this cell (0: interior/Neumann,
// 1: Dirichlet, 2: free-slip).
template <typename T, bool DIAG>
__host__ __device__ __forceinline__ void cell_apply(const T (&u)[4][2][3], const T (&ks)[4], T kcell, bool q0, const T* geo,
                                           T alpha, T beta, T dfac, const int (&bcs)[2], const T (&nrm)[4][3],
                                           T (&out)[4][2][3])
{
    const bool fs_any = (bcs[0] == 2) || (bcs[1] == 2);
    T          uin[4][2][3];
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            T v0 = u[q][s][0], v1 = u[q][s][1], v2 = u[q][s][2];
            if (bcs[s] == 1) {
                v0 = v1 = v2 = T(0);
            } else if (bcs[s] == 2) {
                const T dt = nrm[q][0] * v0 + nrm[q][1] * v1 + nrm[q][2] * v2;
                v0 -= dt * nrm[q][0];
                v1 -= dt * nrm[q][1];
                v2 -= dt * nrm[q][2];
            }
            uin[q][s][0] = v0;
            uin[q][s][1] = v1;
            uin[q][s][2] = v2;
        }

    T ann[4][2];
    if (fs_any) {
#pragma unroll
        for (int q = 0; q < 4; ++q) ann[q][0] = ann[q][1] = T(0);
    }

#pragma unroll
    for (int w = 0; w < 2; ++w) {
        const T* gw = geo + 10 * w;
        const int q0i = wedge_corner(w, 0), q1i = wedge_corner(w, 1), q2i = wedge_corner(w, 2);
        const T   kv  = q0 ? kcell : (ks[q0i] + ks[q1i] + ks[q2i]);
        const T   kw  = kv * gw[9] * dfac;
        T         E1[3], E2[3], E3[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            E1[i] = alpha * gw[i];
            E2[i] = alpha * gw[3 + i];
            E3[i] = beta * gw[6 + i];
        }
        if (!DIAG) {
            T a[3], b[3], D[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const T S0 = uin[q0i][0][c] + uin[q0i][1][c];
                const T S1 = uin[q1i][0][c] + uin[q1i][1][c];
                const T S2 = uin[q2i][0][c] + uin[q2i][1][c];
                a[c]       = S1 - S0;
                b[c]       = S2 - S0;
                D[c]       = (uin[q0i][1][c] - uin[q0i][0][c]) + (uin[q1i][1][c] - uin[q1i][0][c]) +
                       (uin[q2i][1][c] - uin[q2i][0][c]);
            }
            // G[i][j] = d_i u_j
            T G[3][3];
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) G[i][j] = E1[i] * a[j] + E2[i] * b[j] + E3[i] * D[j];
            const T div = G[0][0] + G[1][1] + G[2][2];
            const T k2  = T(2) * kw;
            const T kd  = kw * (T(2) / T(3)) * div;
            const T s00 = k2 * G[0][0] - kd, s11 = k2 * G[1][1] - kd, s22 = k2 * G[2][2] - kd;
            const T s01 = kw * (G[0][1] + G[1][0]), s02 = kw * (G[0][2] + G[2][0]), s12 = kw * (G[1][2] + G[2][1]);
            T       v1[3], v2[3], wv[3];
            v1[0] = s00 * E1[0] + s01 * E1[1] + s02 * E1[2];
            v1[1] = s01 * E1[0] + s11 * E1[1] + s12 * E1[2];
            v1[2] = s02 * E1[0] + s12 * E1[1] + s22 * E1[2];
            v2[0] = s00 * E2[0] + s01 * E2[1] + s02 * E2[2];
            v2[1] = s01 * E2[0] + s11 * E2[1] + s12 * E2[2];
            v2[2] = s02 * E2[0] + s12 * E2[1] + s22 * E2[2];
            wv[0] = s00 * E3[0] + s01 * E3[1] + s02 * E3[2];
            wv[1] = s01 * E3[0] + s11 * E3[1] + s12 * E3[2];
            wv[2] = s02 * E3[0] + s12 * E3[1] + s22 * E3[2];
            const bool bot_on = bcs[0] != 1, top_on = bcs[1] != 1;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const T v0 = -(v1[c] + v2[c]);
                if (bot_on) {
                    out[q0i][0][c] += v0 - wv[c];
                    out[q1i][0][c] += v1[c] - wv[c];
                    out[q2i][0][c] += v2[c] - wv[c];
                }
                if (top_on) {
                    out[q0i][1][c] += v0 + wv[c];
                    out[q1i][1][c] += v1[c] + wv[c];
                    out[q2i][1][c] += v2[c] + wv[c];
                }
            }
        }
        // Diagonal terms: all nodes in DIAG mode, Dirichlet-side nodes otherwise;
        // free-slip normal stiffness Ann on free-slip sides.
        const bool need_diag = DIAG || bcs[0] == 1 || bcs[1] == 1;
        if (need_diag || fs_any) {
#pragma unroll
            for (int s = 0; s < 2; ++s) {
                const bool dir_side = bcs[s] == 1;
                const bool fs_side  = bcs[s] == 2;
                if (!(DIAG || dir_side || fs_side)) continue;
                const T sg = s == 0 ? T(-1) : T(1);
#pragma unroll
                for (int m = 0; m < 3; ++m) {
                    const int q = wedge_corner(w, m);
                    T         g[3];
#pragma unroll
                    for (int i = 0; i < 3; ++i) {
                        const T L = m == 0 ? -(E1[i] + E2[i]) : (m == 1 ? E1[i] : E2[i]);
                        g[i]      = L + sg * E3[i];
                    }
                    const T gg = g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
                    if (fs_side) {
                        const T ng = nrm[q][0] * g[0] + nrm[q][1] * g[1] + nrm[q][2] * g[2];
                        if (!DIAG) {
                            ann[q][s] += kw * (gg + ng * ng * (T(1) / T(3)));
                        } else {
                            T R[3][3];
                            trafo_nt(nrm[q], R);
                            T v[3];
#pragma unroll
                            for (int a_ = 0; a_ < 3; ++a_) {
                                const T Rg = R[a_][0] * g[0] + R[a_][1] * g[1] + R[a_][2] * g[2];
                                const T Rs = R[a_][0] * u[q][s][0] + R[a_][1] * u[q][s][1] + R[a_][2] * u[q][s][2];
                                v[a_]      = kw * (gg + Rg * Rg * (T(1) / T(3))) * Rs;
                            }
#pragma unroll
                            for (int c = 0; c < 3; ++c) out[q][s][c] += R[0][c] * v[0] + R[1][c] * v[1] + R[2][c] * v[2];
                        }
                    } else {
#pragma unroll
                        for (int c = 0; c < 3; ++c)
                            out[q][s][c] += kw * u[q][s][c] * (gg + g[c] * g[c] * (T(1) / T(3)));
                    }
                }
            }
        }
    }

    if (!DIAG && fs_any) {
        // test-side projection and normal stiffness: o <- P o + Ann (n.u) n
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            if (bcs[s] != 2) continue;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const T* n  = nrm[q];
                const T  dt = n[0] * out[q][s][0] + n[1] * out[q][s][1] + n[2] * out[q][s][2];
                const T  un = n[0] * u[q][s][0] + n[1] * u[q][s][1] + n[2] * u[q][s][2];
                const T  cr = ann[q][s] * un - dt;
#pragma unroll
                for (int c = 0; c < 3; ++c) out[q][s][c] += cr * n[c];
            }
        }
    }
}


// ---------------------------------------------------------------------------
// Interior hex cell: both wedges, no boundary treatment. out is assigned.
// ---------------------------------------------------------------------------
template <typename T>
__host__ __device__ __forceinline__ void hex_interior(const T (&u)[4][2][3], const T (&ks)[4], T kcell, bool q0,
                                                      const T* geo, T alpha, T beta, T dfac, T (&out)[4][2][3])
{
    // corner sums and radial differences
    T S[4][3], Dq[4][3];
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            S[q][c]  = u[q][0][c] + u[q][1][c];
            Dq[q][c] = u[q][1][c] - u[q][0][c];
        }
    T v1w[2][3], v2w[2][3], wvw[2][3];
#pragma unroll
    for (int w = 0; w < 2; ++w) {
        const T*  gw  = geo + 10 * w;
        const int q0i = wedge_corner(w, 0), q1i = wedge_corner(w, 1), q2i = wedge_corner(w, 2);
        const T   kv  = q0 ? kcell : (ks[q0i] + ks[q1i] + ks[q2i]);
        const T   kw  = kv * gw[9] * dfac;  // gw[9] = |det M|
        T         E1[3], E2[3], E3[3], a[3], b[3], D[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            E1[i] = alpha * gw[i];
            E2[i] = alpha * gw[3 + i];
            E3[i] = beta * gw[6 + i];
            a[i]  = S[q1i][i] - S[q0i][i];
            b[i]  = S[q2i][i] - S[q0i][i];
            D[i]  = Dq[q0i][i] + Dq[q1i][i] + Dq[q2i][i];
        }
        // symmetric part of G = E1 (x) a + E2 (x) b + E3 (x) D, G[i][j] = d_i u_j
        const T g00 = E1[0] * a[0] + E2[0] * b[0] + E3[0] * D[0];
        const T g11 = E1[1] * a[1] + E2[1] * b[1] + E3[1] * D[1];
        const T g22 = E1[2] * a[2] + E2[2] * b[2] + E3[2] * D[2];
        const T h01 = E1[0] * a[1] + E1[1] * a[0] + E2[0] * b[1] + E2[1] * b[0] + E3[0] * D[1] + E3[1] * D[0];
        const T h02 = E1[0] * a[2] + E1[2] * a[0] + E2[0] * b[2] + E2[2] * b[0] + E3[0] * D[2] + E3[2] * D[0];
        const T h12 = E1[1] * a[2] + E1[2] * a[1] + E2[1] * b[2] + E2[2] * b[1] + E3[1] * D[2] + E3[2] * D[1];
        const T k2  = T(2) * kw;
        const T kd  = kw * (T(2) / T(3)) * (g00 + g11 + g22);
        const T s00 = k2 * g00 - kd, s11 = k2 * g11 - kd, s22 = k2 * g22 - kd;
        const T s01 = kw * h01, s02 = kw * h02, s12 = kw * h12;
        v1w[w][0] = s00 * E1[0] + s01 * E1[1] + s02 * E1[2];
        v1w[w][1] = s01 * E1[0] + s11 * E1[1] + s12 * E1[2];
        v1w[w][2] = s02 * E1[0] + s12 * E1[1] + s22 * E1[2];
        v2w[w][0] = s00 * E2[0] + s01 * E2[1] + s02 * E2[2];
        v2w[w][1] = s01 * E2[0] + s11 * E2[1] + s12 * E2[2];
        v2w[w][2] = s02 * E2[0] + s12 * E2[1] + s22 * E2[2];
        wvw[w][0] = s00 * E3[0] + s01 * E3[1] + s02 * E3[2];
        wvw[w][1] = s01 * E3[0] + s11 * E3[1] + s12 * E3[2];
        wvw[w][2] = s02 * E3[0] + s12 * E3[1] + s22 * E3[2];
    }
    // Nodal outputs sigma g_n per corner: corner 0 is node m = 0 of wedge 0,
    // corner 3 node m = 0 of wedge 1 (lateral part -(v1 + v2)); corner 1 is
    // m = 1 of wedge 0 and m = 2 of wedge 1, corner 2 the reverse. The radial
    // part (wv) enters the bottom node with -1 and the top node with +1.
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const T v120 = v1w[0][c] + v2w[0][c];
        const T v121 = v1w[1][c] + v2w[1][c];
        const T rad  = wvw[0][c] + wvw[1][c];
        const T lat1 = v1w[0][c] + v2w[1][c];
        const T lat2 = v2w[0][c] + v1w[1][c];
        out[0][0][c] = -(v120 + wvw[0][c]);
        out[0][1][c] = wvw[0][c] - v120;
        out[3][0][c] = -(v121 + wvw[1][c]);
        out[3][1][c] = wvw[1][c] - v121;
        out[1][0][c] = lat1 - rad;
        out[1][1][c] = lat1 + rad;
        out[2][0][c] = lat2 - rad;
        out[2][1][c] = lat2 + rad;
    }
}

// Boundary treatment of a hex cell, split around hex_interior:
//   boundary_inputs  : Dirichlet side -> 0, free-slip side -> tangential part
//   boundary_outputs : Dirichlet side -> diagonal rows kw u (|g|^2 + g_c^2/3);
//                      free-slip side -> P out + Ann (n.u) n
// (epsilon_divdiv_kerngen.hpp:1569-1602, 1966-2004, 2108-2160). u_raw is the
// unmodified cell input, nrm the four corner unit normals.
template <typename T>
__host__ __device__ __forceinline__ void boundary_inputs(T (&u)[4][2][3], const int (&bcs)[2], const T (&nrm)[4][3])
{
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        if (bcs[s] == 1) {
#pragma unroll
            for (int q = 0; q < 4; ++q) u[q][s][0] = u[q][s][1] = u[q][s][2] = T(0);
        } else if (bcs[s] == 2) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const T dt = nrm[q][0] * u[q][s][0] + nrm[q][1] * u[q][s][1] + nrm[q][2] * u[q][s][2];
#pragma unroll
                for (int c = 0; c < 3; ++c) u[q][s][c] -= dt * nrm[q][c];
            }
        }
    }
}

template <typename T>
__host__ __device__ __forceinline__ void boundary_outputs(const T (&u)[4][2][3], const T (&ks)[4], T kcell, bool q0,
                                                          const T* geo, T alpha, T beta, T dfac, const int (&bcs)[2],
                                                          const T (&nrm)[4][3], T (&out)[4][2][3])
{
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        if (bcs[s] != 1 && bcs[s] != 2) continue;
        T acc[4][3], ann[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            ann[q] = T(0);
            acc[q][0] = acc[q][1] = acc[q][2] = T(0);
        }
        const T sg = s == 0 ? T(-1) : T(1);
#pragma unroll
        for (int w = 0; w < 2; ++w) {
            const T* gw = geo + 10 * w;
            const T  kv = q0 ? kcell : (ks[wedge_corner(w, 0)] + ks[wedge_corner(w, 1)] + ks[wedge_corner(w, 2)]);
            const T  kw = kv * gw[9] * dfac;
#pragma unroll
            for (int m = 0; m < 3; ++m) {
                const int q = wedge_corner(w, m);
                T         g[3];
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    const T L = m == 0 ? -(gw[i] + gw[3 + i]) : (m == 1 ? gw[i] : gw[3 + i]);
                    g[i]      = alpha * L + sg * beta * gw[6 + i];
                }
                const T gg = g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
                if (bcs[s] == 1) {
#pragma unroll
                    for (int c = 0; c < 3; ++c) acc[q][c] += kw * u[q][s][c] * (gg + g[c] * g[c] * (T(1) / T(3)));
                } else {
                    const T ng = nrm[q][0] * g[0] + nrm[q][1] * g[1] + nrm[q][2] * g[2];
                    ann[q] += kw * (gg + ng * ng * (T(1) / T(3)));
                }
            }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (bcs[s] == 1) {
#pragma unroll
                for (int c = 0; c < 3; ++c) out[q][s][c] = acc[q][c];
            } else {
                const T* n  = nrm[q];
                const T  dt = n[0] * out[q][s][0] + n[1] * out[q][s][1] + n[2] * out[q][s][2];
                const T  un = n[0] * u[q][s][0] + n[1] * u[q][s][1] + n[2] * u[q][s][2];
                const T  cr = ann[q] * un - dt;
#pragma unroll
                for (int c = 0; c < 3; ++c) out[q][s][c] += cr * n[c];
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Per-column boundary coefficients of a boundary cell (side s: 0 bottom, 1 top)
// with radial constants (alpha, beta, dfac) of that cell:
//   Dirichlet: dc[w][m][c] = |det M_w| dfac (|g|^2 + g_c^2 / 3)      18 values
//   free-slip: fc[w][m]    = |det M_w| dfac (|g|^2 + (n.g)^2 / 3)    6 values
// so that at run time the diagonal rows are sum_w kv_w dc u and the normal
// stiffness Ann_q = sum_w kv_w fc (kv_w = coefficient sum of wedge w).
// ---------------------------------------------------------------------------
template <typename T>
__host__ __device__ __forceinline__ void boundary_coefficients(const T* geo, T alpha, T beta, T dfac, int side, int bc,
                                                               const T* nrm /*[4][3]*/, T* out)
{
    const T sg = side == 0 ? T(-1) : T(1);
    for (int w = 0; w < 2; ++w) {
        const T* gw = geo + 10 * w;
        const T  df = gw[9] * dfac;
        for (int m = 0; m < 3; ++m) {
            T g[3];
            for (int i = 0; i < 3; ++i) {
                const T L = m == 0 ? -(gw[i] + gw[3 + i]) : (m == 1 ? gw[i] : gw[3 + i]);
                g[i]      = alpha * L + sg * beta * gw[6 + i];
            }
            const T gg = g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
            if (bc == 1) {
                for (int c = 0; c < 3; ++c) out[(w * 3 + m) * 3 + c] = df * (gg + g[c] * g[c] * (T(1) / T(3)));
            } else {
                const T* n  = nrm + 3 * wedge_corner(w, m);
                const T  ng = n[0] * g[0] + n[1] * g[1] + n[2] * g[2];
                out[w * 3 + m] = df * (gg + ng * ng * (T(1) / T(3)));
            }
        }
    }
}

// Input side of the boundary treatment for side s of a cell: Dirichlet -> 0,
// free-slip -> tangential part (un[q] = n.u of the raw value is returned).
template <typename T>
__host__ __device__ __forceinline__ void side_inputs(T (&u)[4][2][3], int s, int bc, const T* nrm, T (&un)[4])
{
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        if (bc == 1) {
            un[q]      = T(0);
            u[q][s][0] = u[q][s][1] = u[q][s][2] = T(0);
        } else {
            const T* n = nrm + 3 * q;
            un[q]      = n[0] * u[q][s][0] + n[1] * u[q][s][1] + n[2] * u[q][s][2];
#pragma unroll
            for (int c = 0; c < 3; ++c) u[q][s][c] -= un[q] * n[c];
        }
    }
}

// Output side: Dirichlet rows -> diagonal terms of the raw input uraw (side s
// values, [q][c]); free-slip -> P out + Ann (n.u) n.
template <typename T>
__host__ __device__ __forceinline__ void side_outputs(T (&out)[4][2][3], int s, int bc, const T (&ks)[4], T kcell,
                                                      bool q0, const T* coef, const T* nrm, const T (&uraw)[4][3],
                                                      const T (&un)[4])
{
    T kv[2];
#pragma unroll
    for (int w = 0; w < 2; ++w)
        kv[w] = q0 ? kcell : (ks[wedge_corner(w, 0)] + ks[wedge_corner(w, 1)] + ks[wedge_corner(w, 2)]);
    if (bc == 1) {
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int c = 0; c < 3; ++c) out[q][s][c] = T(0);
#pragma unroll
        for (int w = 0; w < 2; ++w)
#pragma unroll
            for (int m = 0; m < 3; ++m) {
                const int q = wedge_corner(w, m);
#pragma unroll
                for (int c = 0; c < 3; ++c) out[q][s][c] += kv[w] * coef[(w * 3 + m) * 3 + c] * uraw[q][c];
            }
    } else {
        T ann[4] = {T(0), T(0), T(0), T(0)};
#pragma unroll
        for (int w = 0; w < 2; ++w)
#pragma unroll
            for (int m = 0; m < 3; ++m) ann[wedge_corner(w, m)] += kv[w] * coef[w * 3 + m];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const T* n  = nrm + 3 * q;
            const T  dt = n[0] * out[q][s][0] + n[1] * out[q][s][1] + n[2] * out[q][s][2];
            const T  cr = ann[q] * un[q] - dt;
#pragma unroll
            for (int c = 0; c < 3; ++c) out[q][s][c] += cr * n[c];
        }
    }
}

}  // namespace tn
