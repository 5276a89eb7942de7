/* CPU oracle for the TERRA-NG Stokes hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, FP64 restatement of the reference's algorithms, used by the tests
 * and by bench.py's CPU-baseline leg to check and time the CUDA product. The
 * product never links or calls this file. Citations are paths inside the
 * reference project (src/terra/...).
 *
 * Compiled with -ffp-contract=off: mesh coordinates must be rounded exactly as
 * the reference's expressions are written.
 */
#include "tn_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define IDX4(nl, nr, d, x, y, r) ((((long)(d) * (nl) + (x)) * (nl) + (y)) * (nr) + (r))
#define LAT(nl, d, x, y) (((long)(d) * (nl) + (x)) * (nl) + (y))

int tno_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

/* ========================================================================== */
/* Mesh                                                                       */
/* ========================================================================== */

/* grid/shell/spherical_shell.hpp:465-604: base nodes and diamond map. */
static void ico_nodes(double n[12][3])
{
    double fifthpi = 0.4 * asin(1.0);
    double w       = 2.0 * acos(1.0 / (2.0 * sin(fifthpi)));
    double cosw    = cos(w);
    double sinw    = sin(w);
    double phi;
    int    k;
    n[0][0] = 0.0; n[0][1] = 0.0; n[0][2] = 1.0;
    n[11][0] = 0.0; n[11][1] = 0.0; n[11][2] = -1.0;
    for (k = 1; k <= 5; k++) {
        phi     = 2.0 * ((double)k - 0.5) * fifthpi;
        n[k][0] = sinw * cos(phi);
        n[k][1] = sinw * sin(phi);
        n[k][2] = cosw;
    }
    for (k = 1; k <= 5; k++) {
        phi         = 2.0 * ((double)k - 1) * fifthpi;
        n[k + 5][0] = sinw * cos(phi);
        n[k + 5][1] = sinw * sin(phi);
        n[k + 5][2] = -cosw;
    }
}

static const int d_node[10][4] = {{0, 5, 6, 1},  {0, 1, 7, 2},  {0, 2, 8, 3},  {0, 3, 9, 4},  {0, 4, 10, 5},
                                  {11, 7, 1, 6}, {11, 8, 2, 7}, {11, 9, 3, 8}, {11, 10, 4, 9}, {11, 6, 5, 10}};

/* compute_node_recursive (spherical_shell.hpp:276-392) with an explicit
 * "computed" flag per node as the memoisation cache. */
typedef struct {
    int     N;
    double* p;     /* (N+1)^2 x 3 */
    char*   done;
} rec_ctx;

static void rec_node(rec_ctx* c, int i, int j, double out[3])
{
    const int N = c->N, ntan = N + 1;
    long      key = (long)i * ntan + j;
    if (c->done[key]) {
        memcpy(out, c->p + 3 * key, 3 * sizeof(double));
        return;
    }
    int l2 = 1, l = 2;
    while (l <= N) {
        if (i % l != 0 || j % l != 0) break;
        l2 *= 2;
        l = 2 * l2;
    }
    double p1[3], p2[3], mid[3];
    if (i % l == 0 && j % l == l2) {
        rec_node(c, i, j - l2, p1);
        rec_node(c, i, j + l2, p2);
    } else if (i % l == l2 && j % l == 0) {
        rec_node(c, i - l2, j, p1);
        rec_node(c, i + l2, j, p2);
    } else {
        rec_node(c, i - l2, j + l2, p1);
        rec_node(c, i + l2, j - l2, p2);
    }
    /* Vec operator+ then normalized() (dense/vec.hpp:58-107) */
    double sum = 0.0, mag;
    int    k;
    for (k = 0; k < 3; k++) mid[k] = p1[k] + p2[k];
    for (k = 0; k < 3; k++) sum += mid[k] * mid[k];
    mag = sqrt(sum);
    if (mag > 1e-15)
        for (k = 0; k < 3; k++) mid[k] /= mag;
    memcpy(c->p + 3 * key, mid, 3 * sizeof(double));
    c->done[key] = 1;
    memcpy(out, mid, 3 * sizeof(double));
}

int tno_unit_sphere_coords(int lat_level, double* out)
{
    if (lat_level < 0 || lat_level > 10) return -1;
    double nodes[12][3];
    ico_nodes(nodes);
    const int N = 1 << lat_level, ntan = N + 1;
    rec_ctx   c;
    c.N    = N;
    c.p    = (double*)malloc(sizeof(double) * 3 * ntan * ntan);
    c.done = (char*)malloc((size_t)ntan * ntan);
    for (int d = 0; d < 10; d++) {
        int L = d < 5 ? 1 : 3, R = d < 5 ? 3 : 1;
        memset(c.done, 0, (size_t)ntan * ntan);
        const int corner_key[4] = {0, N * ntan, N * ntan + N, N};   /* p00, pN0, pNN, p0N */
        const int corner_node[4] = {d_node[d][0], d_node[d][L], d_node[d][2], d_node[d][R]};
        for (int q = 0; q < 4; q++) {
            memcpy(c.p + 3 * corner_key[q], nodes[corner_node[q]], 3 * sizeof(double));
            c.done[corner_key[q]] = 1;
        }
        for (int i = 0; i < ntan; i++)
            for (int j = 0; j < ntan; j++) {
                double v[3];
                rec_node(&c, i, j, v);
                memcpy(out + 3 * LAT(ntan, d, i, j), v, 3 * sizeof(double));
            }
    }
    free(c.p);
    free(c.done);
    return 0;
}

int tno_uniform_radii(double r_min, double r_max, int num_shells, double* out)
{
    if (num_shells < 2 || r_min >= r_max) return -1;
    double r_step = (r_max - r_min) / (num_shells - 1);
    for (int i = 0; i < num_shells; i++) out[i] = r_min + i * r_step;
    out[num_shells - 1] = r_max;
    return 0;
}

/* Union-find over the diamond face equivalences stated at
 * spherical_shell.hpp:1153-1176 (one subdomain per diamond):
 *   d_k(0, t)   = d_{k+1}(t, 0)        within each hemisphere ring
 *   d_k(t, end) = d_{k+5}(end, end-t)  north -> south
 *   d_{k+5}(t, end) = d_{k+1}(end, end-t)  south -> north        */
static int uf_find(int* p, int a)
{
    while (p[a] != a) {
        p[a] = p[p[a]];
        a    = p[a];
    }
    return a;
}
static void uf_union(int* p, int a, int b)
{
    a = uf_find(p, a);
    b = uf_find(p, b);
    if (a != b) {
        if (a < b) p[b] = a; else p[a] = b;
    }
}

int tno_duplicate_classes(int lat_level, int32_t* class_of_lat)
{
    const int nl = (1 << lat_level) + 1, E = nl - 1;
    const int n  = 10 * nl * nl;
    int*      p  = (int*)malloc(sizeof(int) * n);
    int*      cnt = (int*)calloc(n, sizeof(int));
    for (int i = 0; i < n; i++) p[i] = i;
    for (int k = 0; k < 5; k++)
        for (int t = 0; t <= E; t++) {
            uf_union(p, LAT(nl, k, 0, t), LAT(nl, (k + 1) % 5, t, 0));
            uf_union(p, LAT(nl, 5 + k, 0, t), LAT(nl, 5 + (k + 1) % 5, t, 0));
            uf_union(p, LAT(nl, k, t, E), LAT(nl, k + 5, E, E - t));
            uf_union(p, LAT(nl, k + 5, t, E), LAT(nl, (k + 1) % 5, E, E - t));
        }
    for (int i = 0; i < n; i++) cnt[uf_find(p, i)]++;
    int* id     = (int*)malloc(sizeof(int) * n);
    int  nclass = 0;
    for (int i = 0; i < n; i++) id[i] = -1;
    for (int i = 0; i < n; i++) {
        int root = uf_find(p, i);
        if (cnt[root] < 2) {
            class_of_lat[i] = -1;
            continue;
        }
        if (id[root] < 0) id[root] = nclass++;
        class_of_lat[i] = id[root];
    }
    free(p);
    free(cnt);
    free(id);
    return nclass;
}

/* grid/bit_masks.hpp:27-85: owner = copy in the subdomain with the smallest
 * global id, which for one subdomain per diamond is the smallest diamond id. */
int tno_ownership(int lat_level, uint8_t* owned_lat)
{
    const int nl = (1 << lat_level) + 1;
    const int n  = 10 * nl * nl;
    int32_t*  cls = (int32_t*)malloc(sizeof(int32_t) * n);
    int       nc  = tno_duplicate_classes(lat_level, cls);
    int*      first = (int*)malloc(sizeof(int) * (nc > 0 ? nc : 1));
    for (int c = 0; c < nc; c++) first[c] = -1;
    for (int i = 0; i < n; i++) {
        if (cls[i] < 0) {
            owned_lat[i] = 1;
            continue;
        }
        if (first[cls[i]] < 0) {   /* lateral index order == diamond order */
            first[cls[i]] = i;
            owned_lat[i]  = 1;
        } else
            owned_lat[i] = 0;
    }
    free(cls);
    free(first);
    return 0;
}

int tno_boundary_mask(int nl, int nr, uint8_t* mask)
{
    for (int d = 0; d < 10; d++)
        for (int x = 0; x < nl; x++)
            for (int y = 0; y < nl; y++)
                for (int r = 0; r < nr; r++) {
                    uint8_t f = 1; /* INNER */
                    if (r == 0) f = 2 | 4; /* CMB */
                    if (r == nr - 1) f = 2 | 8; /* SURFACE (overwrites, as the reference sets it last) */
                    mask[IDX4(nl, nr, d, x, y, r)] = f;
                }
    return 0;
}

/* ========================================================================== */
/* Wedge element helpers (fe/wedge/integrands.hpp, kernel_helpers.hpp)        */
/* ========================================================================== */

/* WEDGE_NODE_OFF: node offsets of the two wedges of a hex cell
 * (kernel_helpers.hpp:291-312). */
static const int WOFF[2][6][3] = {{{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {0, 1, 1}},
                                  {{1, 1, 0}, {0, 1, 0}, {1, 0, 0}, {1, 1, 1}, {0, 1, 1}, {1, 0, 1}}};

static double shape_rad(int node, double zeta)
{
    double N_rad[2] = {0.5 * (1 - zeta), 0.5 * (1 + zeta)};
    return N_rad[node / 3];
}
static double shape_lat(int node, double xi, double eta)
{
    double N_lat[3] = {1.0 - xi - eta, xi, eta};
    return N_lat[node % 3];
}
static double shape(int node, const double q[3]) { return shape_lat(node, q[0], q[1]) * shape_rad(node, q[2]); }
static void grad_shape(int node, const double q[3], double g[3])
{
    static const double gxi[3] = {-1.0, 1.0, 0.0}, geta[3] = {-1.0, 0.0, 1.0}, grad_rad[2] = {-0.5, 0.5};
    g[0] = gxi[node % 3] * shape_rad(node, q[2]);
    g[1] = geta[node % 3] * shape_rad(node, q[2]);
    g[2] = shape_lat(node, q[0], q[1]) * grad_rad[node / 3];
}

/* jac() (integrands.hpp:610-640): J = jac_lat * diag(r, r, dr/2). Row-major J[i][j]. */
static void jacobian(const double p[3][3], double r1, double r2, const double q[3], double J[3][3])
{
    double r      = r1 + 0.5 * (r2 - r1) * (1 + q[2]);
    double grad_r = 0.5 * (r2 - r1);
    double col[3][3];
    for (int i = 0; i < 3; i++) {
        col[0][i] = p[1][i] - p[0][i];
        col[1][i] = p[2][i] - p[0][i];
        col[2][i] = (1 - q[0] - q[1]) * p[0][i] + q[0] * p[1][i] + q[1] * p[2][i];
    }
    double s[3] = {r, r, grad_r};
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) J[i][j] = col[j][i] * s[j];
}

/* Mat::det / inv_transposed (dense/mat.hpp:240-335). */
static double det3(const double a[3][3])
{
    return a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) - a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) +
           a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
}
static void inv_transposed(const double a[3][3], double d, double r[3][3])
{
    double id = 1.0 / d;
    r[0][0]   = (a[1][1] * a[2][2] - a[1][2] * a[2][1]) * id;
    r[0][1]   = -(a[1][0] * a[2][2] - a[1][2] * a[2][0]) * id;
    r[0][2]   = (a[1][0] * a[2][1] - a[1][1] * a[2][0]) * id;
    r[1][0]   = -(a[0][1] * a[2][2] - a[0][2] * a[2][1]) * id;
    r[1][1]   = (a[0][0] * a[2][2] - a[0][2] * a[2][0]) * id;
    r[1][2]   = -(a[0][0] * a[2][1] - a[0][1] * a[2][0]) * id;
    r[2][0]   = (a[0][1] * a[1][2] - a[0][2] * a[1][1]) * id;
    r[2][1]   = -(a[0][0] * a[1][2] - a[0][2] * a[1][0]) * id;
    r[2][2]   = (a[0][0] * a[1][1] - a[0][1] * a[1][0]) * id;
}

/* wedge_surface_physical_coords (kernel_helpers.hpp:25-56). */
static void wedge_surface(const double* coords, int nl, int d, int x, int y, double ws[2][3][3])
{
    const double* q00 = coords + 3 * LAT(nl, d, x, y);
    const double* q10 = coords + 3 * LAT(nl, d, x + 1, y);
    const double* q01 = coords + 3 * LAT(nl, d, x, y + 1);
    const double* q11 = coords + 3 * LAT(nl, d, x + 1, y + 1);
    for (int i = 0; i < 3; i++) {
        ws[0][0][i] = q00[i]; ws[0][1][i] = q10[i]; ws[0][2][i] = q01[i];
        ws[1][0][i] = q11[i]; ws[1][1][i] = q01[i]; ws[1][2][i] = q10[i];
    }
}

/* normal-tangential frame (linalg/trafo/local_basis_trafo_normal_tangential.hpp:34-76). */
static void vnormalized(const double a[3], double o[3])
{
    double s = 0.0;
    for (int i = 0; i < 3; i++) s += a[i] * a[i];
    double m = sqrt(s);
    for (int i = 0; i < 3; i++) o[i] = a[i];
    if (m > 1e-15)
        for (int i = 0; i < 3; i++) o[i] /= m;
}
static void cross(const double a[3], const double b[3], double o[3])
{
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}
static void trafo_nt(const double nin[3], double R[3][3])
{
    double n[3], ref[3] = {0, 0, 0}, t1[3], t2[3], tmp[3];
    vnormalized(nin, n);
    double ax = fabs(n[0]), ay = fabs(n[1]), az = fabs(n[2]);
    if (ax <= ay && ax <= az) ref[0] = 1;
    else if (ay <= ax && ay <= az) ref[1] = 1;
    else ref[2] = 1;
    cross(ref, n, tmp);
    vnormalized(tmp, t1);
    double s = 0;
    for (int i = 0; i < 3; i++) s += t1[i] * t1[i];
    if (sqrt(s) < 1e-15) {
        double a[3] = {n[1], -n[0], 0.0};
        vnormalized(a, t1);
    }
    cross(n, t1, tmp);
    vnormalized(tmp, t2);
    for (int i = 0; i < 3; i++) {
        R[0][i] = n[i];
        R[1][i] = t1[i];
        R[2][i] = t2[i];
    }
}

/* Felippa 1x1 point and weight (quadrature.hpp:32-46). */
static const double QP[3] = {1.0 / 3.0, 1.0 / 3.0, 0.0};
static const double QW    = 1.0;

/* k_eval of a wedge: nodal interpolation at the quadrature point or the Q0 value. */
static double wedge_k(const tno_op* op, int d, int x, int y, int r, int w)
{
    if (op->k_q0) return op->k_q0[IDX4(op->nl - 1, op->nr - 1, d, x, y, r)];
    double kv = 0.0;
    for (int n = 0; n < 6; n++)
        kv += shape(n, QP) * op->k[IDX4(op->nl, op->nr, d, x + WOFF[w][n][0], y + WOFF[w][n][1], r + WOFF[w][n][2])];
    return kv;
}

/* assemble_local_matrix (epsilon_divdiv_kerngen.hpp:2315-2392): dimension-wise
 * ordering, A[(i + 6 dimi) * 18 + (j + 6 dimj)]. */
static void local_matrix(const tno_op* op, int d, int x, int y, int r, int w, double A[18 * 18])
{
    double ws[2][3][3], J[3][3], JiT[3][3], g[6][3];
    wedge_surface(op->coords, op->nl, d, x, y, ws);
    double r1 = op->radii[r], r2 = op->radii[r + 1];
    jacobian(ws[w], r1, r2, QP, J);
    double det = det3(J);
    inv_transposed(J, det, JiT);
    double kv  = wedge_k(op, d, x, y, r, w);
    double jkw = QW * kv * fabs(det);
    for (int n = 0; n < 6; n++) {
        double gr[3];
        grad_shape(n, QP, gr);
        for (int a = 0; a < 3; a++) g[n][a] = JiT[a][0] * gr[0] + JiT[a][1] * gr[1] + JiT[a][2] * gr[2];
    }
    memset(A, 0, sizeof(double) * 324);
    for (int di = 0; di < 3; di++)
        for (int dj = 0; dj < 3; dj++)
            for (int i = 0; i < 6; i++)
                for (int j = 0; j < 6; j++) {
                    /* symgrad(n, dim)_{ab} = (g_a delta_{b,dim} + g_b delta_{a,dim}) / 2 */
                    double dc = 0.0;
                    for (int a = 0; a < 3; a++)
                        for (int b = 0; b < 3; b++) {
                            double si = 0.5 * ((b == di ? g[i][a] : 0.0) + (a == di ? g[i][b] : 0.0));
                            double sj = 0.5 * ((b == dj ? g[j][a] : 0.0) + (a == dj ? g[j][b] : 0.0));
                            dc += sj * si;
                        }
                    A[(i + 6 * di) * 18 + (j + 6 * dj)] += jkw * (2 * dc - 2.0 / 3.0 * g[j][dj] * g[i][di]);
                }
}

int tno_epsdivdiv_local_matrix(const tno_op* op, int d, int x, int y, int r, int wedge, double* A)
{
    local_matrix(op, d, x, y, r, wedge, A);
    return 0;
}

static void physical_coords(const tno_op* op, int d, int x, int y, int r, double out[3])
{
    const double* c = op->coords + 3 * LAT(op->nl, d, x, y);
    for (int i = 0; i < 3; i++) out[i] = c[i] * op->radii[r];
}

/* Slow-path cell apply (epsilon_divdiv_kerngen.hpp:1013-1242) given the two
 * (unmasked) wedge matrices. Adds into dst. */
static void slow_cell_local(const tno_op* op, int d, int x, int y, int r, double A[2][324], const double* const* src,
                            double outw[2][18])
{
    const int nl = op->nl, nr = op->nr;
    int       at_cmb = (r == 0), at_surface = (r + 1 == nr - 1);
    double    s[2][18], mask[324], R[2][324];
    int       freeslip = 0;
    for (int w = 0; w < 2; w++)
        for (int dim = 0; dim < 3; dim++)
            for (int n = 0; n < 6; n++)
                s[w][dim * 6 + n] =
                    src[dim][IDX4(nl, nr, d, x + WOFF[w][n][0], y + WOFF[w][n][1], r + WOFF[w][n][2])];
    for (int i = 0; i < 324; i++) mask[i] = 1.0;
    if (at_cmb || at_surface) {
        int bcf = at_cmb ? op->bc_cmb : op->bc_surface;
        if (bcf == 1) {
            for (int di = 0; di < 3; di++)
                for (int dj = 0; dj < 3; dj++)
                    for (int i = 0; i < 6; i++)
                        for (int j = 0; j < 6; j++)
                            if ((at_cmb && ((di == dj && i != j && (i < 3 || j < 3)) || (di != dj && (i < 3 || j < 3)))) ||
                                (at_surface &&
                                 ((di == dj && i != j && (i >= 3 || j >= 3)) || (di != dj && (i >= 3 || j >= 3)))))
                                mask[(i + di * 6) * 18 + (j + dj * 6)] = 0.0;
        } else if (bcf == 2) {
            static const int ox[2][3] = {{0, 1, 0}, {1, 0, 1}}, oy[2][3] = {{0, 0, 1}, {1, 1, 0}};
            freeslip = 1;
            for (int w = 0; w < 2; w++) {
                double At[324], sn[18], tmp[324];
                /* dimension-wise -> node-wise reordering */
                for (int di = 0; di < 3; di++)
                    for (int i = 0; i < 6; i++)
                        for (int dj = 0; dj < 3; dj++)
                            for (int j = 0; j < 6; j++)
                                At[(i * 3 + di) * 18 + (j * 3 + dj)] = A[w][(i + di * 6) * 18 + (j + dj * 6)];
                for (int dim = 0; dim < 3; dim++)
                    for (int n = 0; n < 6; n++) sn[n * 3 + dim] = s[w][n + dim * 6];
                memset(R[w], 0, sizeof(double) * 324);
                for (int i = 0; i < 18; i++) R[w][i * 18 + i] = 1.0;
                for (int b = 0; b < 3; b++) {
                    double nrm[3], Ri[3][3];
                    physical_coords(op, d, x + ox[w][b], y + oy[w][b], r + (at_cmb ? 0 : 1), nrm);
                    trafo_nt(nrm, Ri);
                    int off = at_cmb ? 0 : 9;
                    for (int a = 0; a < 3; a++)
                        for (int c = 0; c < 3; c++) R[w][(off + b * 3 + a) * 18 + off + b * 3 + c] = Ri[a][c];
                }
                /* A = R At R^T */
                for (int i = 0; i < 18; i++)
                    for (int j = 0; j < 18; j++) {
                        double acc = 0;
                        for (int k = 0; k < 18; k++) acc += R[w][i * 18 + k] * At[k * 18 + j];
                        tmp[i * 18 + j] = acc;
                    }
                for (int i = 0; i < 18; i++)
                    for (int j = 0; j < 18; j++) {
                        double acc = 0;
                        for (int k = 0; k < 18; k++) acc += tmp[i * 18 + k] * R[w][j * 18 + k];
                        A[w][i * 18 + j] = acc;
                    }
                for (int i = 0; i < 18; i++) {
                    double acc = 0;
                    for (int k = 0; k < 18; k++) acc += R[w][i * 18 + k] * sn[k];
                    s[w][i] = acc;
                }
                int ns = at_surface ? 3 : 0, ne = at_surface ? 6 : 3;
                for (int nn = ns; nn < ne; nn++) {
                    int idx = nn * 3;
                    for (int k = 0; k < 18; k++)
                        if (k != idx) {
                            mask[idx * 18 + k] = 0.0;
                            mask[k * 18 + idx] = 0.0;
                        }
                }
            }
        }
    }
    for (int w = 0; w < 2; w++) {
        double out[18];
        for (int i = 0; i < 324; i++) A[w][i] *= mask[i];
        for (int i = 0; i < 18; i++) {
            double acc = 0;
            if (op->diagonal)
                acc = A[w][i * 18 + i] * s[w][i];
            else
                for (int j = 0; j < 18; j++) acc += A[w][i * 18 + j] * s[w][j];
            out[i] = acc;
        }
        if (freeslip) {
            double o2[18];
            for (int i = 0; i < 18; i++) {
                double acc = 0;
                for (int k = 0; k < 18; k++) acc += R[w][k * 18 + i] * out[k];
                o2[i] = acc;
            }
            for (int dim = 0; dim < 3; dim++)
                for (int n = 0; n < 6; n++) out[n + dim * 6] = o2[n * 3 + dim];
        }
        for (int i = 0; i < 18; i++) outw[w][i] = out[i];
    }
}

/* Slow-path cell apply: adds the cell's outputs into dst. */
static void slow_cell(const tno_op* op, int d, int x, int y, int r, double A[2][324], const double* const* src,
                      double* const* dst)
{
    const int nl = op->nl, nr = op->nr;
    double    outw[2][18];
    slow_cell_local(op, d, x, y, r, A, src, outw);
    for (int w = 0; w < 2; w++)
        for (int dim = 0; dim < 3; dim++)
            for (int n = 0; n < 6; n++)
                dst[dim][IDX4(nl, nr, d, x + WOFF[w][n][0], y + WOFF[w][n][1], r + WOFF[w][n][2])] +=
                    outw[w][dim * 6 + n];
}

/* Cell loops are split into two x-parity sweeps so that concurrent threads
 * never touch the same node; results do not depend on the thread count. */
#define CELL_LOOP_BEGIN(nl, nr)                                                   \
    for (int parity = 0; parity < 2; parity++) {                                  \
        _Pragma("omp parallel for collapse(2) schedule(static)")                  \
        for (int d = 0; d < 10; d++)                                              \
            for (int xh = 0; xh < ((nl) - 1 + 1 - parity) / 2; xh++) {            \
                int x = 2 * xh + parity;                                          \
                for (int y = 0; y < (nl) - 1; y++)                                \
                    for (int r = 0; r < (nr) - 1; r++) {
#define CELL_LOOP_END \
    }                 \
    }                 \
    }

static void zero_vec(double* const* v, int ncomp, long n)
{
    for (int c = 0; c < ncomp; c++) memset(v[c], 0, sizeof(double) * n);
}

int tno_epsdivdiv_slow(const tno_op* op, const double* const* src, double* const* dst)
{
    const int nl = op->nl, nr = op->nr;
    zero_vec(dst, 3, 10L * nl * nl * nr);
    CELL_LOOP_BEGIN(nl, nr)
    double A[2][324];
    local_matrix(op, d, x, y, r, 0, A[0]);
    local_matrix(op, d, x, y, r, 1, A[1]);
    slow_cell(op, d, x, y, r, A, src, dst);
    CELL_LOOP_END
    return 0;
}

int tno_epsdivdiv_stored(const tno_op* op, const double* mats, const double* const* src, double* const* dst)
{
    const int nl = op->nl, nr = op->nr;
    zero_vec(dst, 3, 10L * nl * nl * nr);
    CELL_LOOP_BEGIN(nl, nr)
    double A[2][324];
    long   c = IDX4(nl - 1, nr - 1, d, x, y, r);
    memcpy(A[0], mats + (c * 2 + 0) * 324, sizeof(double) * 324);
    memcpy(A[1], mats + (c * 2 + 1) * 324, sizeof(double) * 324);
    slow_cell(op, d, x, y, r, A, src, dst);
    CELL_LOOP_END
    return 0;
}

/* -------------------------------------------------------------------------- */
/* Fast paths, restated from the reference's fused kernels.                   */
/* -------------------------------------------------------------------------- */

static const double ONE_THIRD = 1.0 / 3.0, ONE_SIXTH = 1.0 / 6.0, NEG_TWO_THIRDS = -0.66666666666666663;
static const double dN_ref[6][3] = {{-0.5, -0.5, -1.0 / 6.0}, {0.5, 0.0, -1.0 / 6.0}, {0.0, 0.5, -1.0 / 6.0},
                                    {-0.5, -0.5, 1.0 / 6.0},  {0.5, 0.0, 1.0 / 6.0},  {0.0, 0.5, 1.0 / 6.0}};

/* Jacobian at the centroid and its inverse-transposed, written out as in
 * epsilon_divdiv_kerngen.hpp:1437-1470. Returns det. */
static double fast_jac(const double* c0, const double* c1, const double* c2, double r0, double r1, double I[3][3])
{
    double half_dr = 0.5 * (r1 - r0), r_mid = 0.5 * (r0 + r1), J[3][3];
    for (int i = 0; i < 3; i++) {
        J[i][0] = r_mid * (-c0[i] + c1[i]);
        J[i][1] = r_mid * (-c0[i] + c2[i]);
        J[i][2] = half_dr * (ONE_THIRD * (c0[i] + c1[i] + c2[i]));
    }
    double det = J[0][0] * J[1][1] * J[2][2] - J[0][0] * J[1][2] * J[2][1] - J[0][1] * J[1][0] * J[2][2] +
                 J[0][1] * J[1][2] * J[2][0] + J[0][2] * J[1][0] * J[2][1] - J[0][2] * J[1][1] * J[2][0];
    double id = 1.0 / det;
    I[0][0]   = id * (J[1][1] * J[2][2] - J[1][2] * J[2][1]);
    I[0][1]   = id * (-J[1][0] * J[2][2] + J[1][2] * J[2][0]);
    I[0][2]   = id * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
    I[1][0]   = id * (-J[0][1] * J[2][2] + J[0][2] * J[2][1]);
    I[1][1]   = id * (J[0][0] * J[2][2] - J[0][2] * J[2][0]);
    I[1][2]   = id * (-J[0][0] * J[2][1] + J[0][1] * J[2][0]);
    I[2][0]   = id * (J[0][1] * J[1][2] - J[0][2] * J[1][1]);
    I[2][1]   = id * (-J[0][0] * J[1][2] + J[0][2] * J[1][0]);
    I[2][2]   = id * (J[0][0] * J[1][1] - J[0][1] * J[1][0]);
    return det;
}

static void phys_grad(double I[3][3], int n, double g[3])
{
    for (int a = 0; a < 3; a++) g[a] = I[a][0] * dN_ref[n][0] + I[a][1] * dN_ref[n][1] + I[a][2] * dN_ref[n][2];
}

int tno_epsdivdiv_fast(const tno_op* op, const double* const* src, double* const* dst)
{
    const int nl = op->nl, nr = op->nr;
    zero_vec(dst, 3, 10L * nl * nl * nr);
    static const int WTU[2][6] = {{0, 1, 2, 3, 4, 5}, {6, 2, 1, 7, 5, 4}};
    /* unique hex corner u -> (dx, dy, dr) */
    static const int UOFF[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {0, 1, 1}, {1, 1, 0}, {1, 1, 1}};
    static const int CORNER_OFF[4][2] = {{0, 0}, {1, 0}, {0, 1}, {1, 1}};
    static const int CMB_C2U[4] = {0, 1, 2, 6}, SURF_C2U[4] = {3, 4, 5, 7};
    static const int N2C[2][3] = {{0, 1, 2}, {3, 2, 1}};
    const int diag = op->diagonal;
    CELL_LOOP_BEGIN(nl, nr)
    const int at_cmb = (r == 0), at_surface = (r + 1 == nr - 1);
    const int cmb_fs = at_cmb && op->bc_cmb == 2, surf_fs = at_surface && op->bc_surface == 2;
    const int cmb_di = at_cmb && op->bc_cmb == 1, surf_di = at_surface && op->bc_surface == 1;
    const int cmb_shift = (cmb_di && !diag) ? 3 : 0, surf_shift = (surf_di && !diag) ? 3 : 0;
    double    dst8[3][8];
    double    Ann_c[4] = {0, 0, 0, 0}, Ann_s[4] = {0, 0, 0, 0};
    double    nrm[4][3];
    memset(dst8, 0, sizeof(dst8));
    for (int c = 0; c < 4; c++) {
        const double* cc = op->coords + 3 * LAT(nl, d, x + CORNER_OFF[c][0], y + CORNER_OFF[c][1]);
        double        n2 = cc[0] * cc[0] + cc[1] * cc[1] + cc[2] * cc[2];
        double        in = 1.0 / sqrt(n2);
        for (int i = 0; i < 3; i++) nrm[c][i] = cc[i] * in;
    }
    for (int w = 0; w < 2; w++) {
        const double* v0 = op->coords + 3 * LAT(nl, d, x + WOFF[w][0][0], y + WOFF[w][0][1]);
        const double* v1 = op->coords + 3 * LAT(nl, d, x + WOFF[w][1][0], y + WOFF[w][1][1]);
        const double* v2 = op->coords + 3 * LAT(nl, d, x + WOFF[w][2][0], y + WOFF[w][2][1]);
        double        k_eval;
        if (op->k_q0)
            k_eval = op->k_q0[IDX4(nl - 1, nr - 1, d, x, y, r)];
        else {
            double ks = 0;
            for (int n = 0; n < 6; n++)
                ks += op->k[IDX4(nl, nr, d, x + WOFF[w][n][0], y + WOFF[w][n][1], r + WOFF[w][n][2])];
            k_eval = ONE_SIXTH * ks;
        }
        double I[3][3];
        double det = fast_jac(v0, v1, v2, op->radii[r], op->radii[r + 1], I);
        double kwJ = k_eval * fabs(det);
        double s[6][3], g[6][3];
        for (int n = 0; n < 6; n++) {
            long id = IDX4(nl, nr, d, x + WOFF[w][n][0], y + WOFF[w][n][1], r + WOFF[w][n][2]);
            for (int c = 0; c < 3; c++) s[n][c] = src[c][id];
            phys_grad(I, n, g[n]);
        }
        if (!diag) {
            double gu00 = 0, gu10 = 0, gu11 = 0, gu20 = 0, gu21 = 0, gu22 = 0, div_u = 0;
            for (int n = cmb_shift; n < 6 - surf_shift; n++) {
                double s0 = s[n][0], s1 = s[n][1], s2 = s[n][2];
                if ((cmb_fs && n < 3) || (surf_fs && n >= 3)) {
                    const double* nn = nrm[n < 3 ? N2C[w][n] : N2C[w][n - 3]];
                    double        dt = nn[0] * s0 + nn[1] * s1 + nn[2] * s2;
                    s0 -= dt * nn[0];
                    s1 -= dt * nn[1];
                    s2 -= dt * nn[2];
                }
                const double* gg = g[n];
                gu00 += gg[0] * s0;
                gu11 += gg[1] * s1;
                gu22 += gg[2] * s2;
                gu10 += 0.5 * (gg[1] * s0 + gg[0] * s1);
                gu20 += 0.5 * (gg[2] * s0 + gg[0] * s2);
                gu21 += 0.5 * (gg[2] * s1 + gg[1] * s2);
                div_u += gg[0] * s0 + gg[1] * s1 + gg[2] * s2;
            }
            for (int n = cmb_shift; n < 6 - surf_shift; n++) {
                const double* gg  = g[n];
                int           uid = WTU[w][n];
                dst8[0][uid] += kwJ * (2.0 * (gg[0] * gu00 + gg[1] * gu10 + gg[2] * gu20) + NEG_TWO_THIRDS * gg[0] * div_u);
                dst8[1][uid] += kwJ * (2.0 * (gg[0] * gu10 + gg[1] * gu11 + gg[2] * gu21) + NEG_TWO_THIRDS * gg[1] * div_u);
                dst8[2][uid] += kwJ * (2.0 * (gg[0] * gu20 + gg[1] * gu21 + gg[2] * gu22) + NEG_TWO_THIRDS * gg[2] * div_u);
                if ((cmb_fs && n < 3) || (surf_fs && n >= 3)) {
                    int           corner = n < 3 ? N2C[w][n] : N2C[w][n - 3];
                    const double* nn     = nrm[corner];
                    double        g2     = gg[0] * gg[0] + gg[1] * gg[1] + gg[2] * gg[2];
                    double        ng     = nn[0] * gg[0] + nn[1] * gg[1] + nn[2] * gg[2];
                    if (n < 3) Ann_c[corner] += kwJ * (g2 + ONE_THIRD * ng * ng);
                    else Ann_s[corner] += kwJ * (g2 + ONE_THIRD * ng * ng);
                }
            }
        }
        if (diag || cmb_di || surf_di) {
            for (int n = surf_shift; n < 6 - cmb_shift; n++) {
                if (diag && ((cmb_fs && n < 3) || (surf_fs && n >= 3))) continue;
                const double* gg  = g[n];
                double        g2  = gg[0] * gg[0] + gg[1] * gg[1] + gg[2] * gg[2];
                int           uid = WTU[w][n];
                for (int c = 0; c < 3; c++) dst8[c][uid] += kwJ * s[n][c] * (g2 + ONE_THIRD * gg[c] * gg[c]);
            }
            if (diag) {
                for (int side = 0; side < 2; side++) {
                    if (!(side == 0 ? cmb_fs : surf_fs)) continue;
                    for (int ni = 0; ni < 3; ni++) {
                        int           n      = ni + 3 * side;
                        int           corner = N2C[w][ni];
                        const double* nn     = nrm[corner];
                        double        Rr[3][3];
                        trafo_nt(nn, Rr);
                        const double* gg = g[n];
                        double        g2 = gg[0] * gg[0] + gg[1] * gg[1] + gg[2] * gg[2];
                        long id = IDX4(nl, nr, d, x + CORNER_OFF[corner][0], y + CORNER_OFF[corner][1], r + side);
                        double sv[3] = {src[0][id], src[1][id], src[2][id]}, Rg[3], Rs[3], v[3];
                        for (int a = 0; a < 3; a++) {
                            Rg[a] = Rr[a][0] * gg[0] + Rr[a][1] * gg[1] + Rr[a][2] * gg[2];
                            Rs[a] = Rr[a][0] * sv[0] + Rr[a][1] * sv[1] + Rr[a][2] * sv[2];
                        }
                        for (int a = 0; a < 3; a++) v[a] = kwJ * (g2 + ONE_THIRD * Rg[a] * Rg[a]) * Rs[a];
                        int u = WTU[w][n];
                        for (int c = 0; c < 3; c++) dst8[c][u] += Rr[0][c] * v[0] + Rr[1][c] * v[1] + Rr[2][c] * v[2];
                    }
                }
            }
        }
    }
    if (!diag) {
        for (int side = 0; side < 2; side++) {
            if (!(side == 0 ? cmb_fs : surf_fs)) continue;
            const int* c2u = side == 0 ? CMB_C2U : SURF_C2U;
            double*    Ann = side == 0 ? Ann_c : Ann_s;
            for (int c = 0; c < 4; c++) {
                const double* nn = nrm[c];
                int           u  = c2u[c];
                double        dt = nn[0] * dst8[0][u] + nn[1] * dst8[1][u] + nn[2] * dst8[2][u];
                for (int i = 0; i < 3; i++) dst8[i][u] -= dt * nn[i];
                long   id = IDX4(nl, nr, d, x + CORNER_OFF[c][0], y + CORNER_OFF[c][1], r + side);
                double un = nn[0] * src[0][id] + nn[1] * src[1][id] + nn[2] * src[2][id];
                for (int i = 0; i < 3; i++) dst8[i][u] += Ann[c] * un * nn[i];
            }
        }
    }
    for (int u = 0; u < 8; u++) {
        long id = IDX4(nl, nr, d, x + UOFF[u][0], y + UOFF[u][1], r + UOFF[u][2]);
        for (int c = 0; c < 3; c++) dst[c][id] += dst8[c][u];
    }
    CELL_LOOP_END
    return 0;
}

/* ========================================================================== */
/* Interface sum, dots                                                        */
/* ========================================================================== */

int tno_interface_sum(int lat_level, int nr, int ncomp, double* const* v)
{
    const int nl = (1 << lat_level) + 1;
    const int n  = 10 * nl * nl;
    int32_t*  cls = (int32_t*)malloc(sizeof(int32_t) * n);
    int       nc  = tno_duplicate_classes(lat_level, cls);
    double*   acc = (double*)malloc(sizeof(double) * (size_t)(nc > 0 ? nc : 1) * nr);
    for (int c = 0; c < ncomp; c++) {
        memset(acc, 0, sizeof(double) * (size_t)(nc > 0 ? nc : 1) * nr);
        for (int i = 0; i < n; i++)
            if (cls[i] >= 0)
                for (int r = 0; r < nr; r++) acc[(long)cls[i] * nr + r] += v[c][(long)i * nr + r];
        for (int i = 0; i < n; i++)
            if (cls[i] >= 0)
                for (int r = 0; r < nr; r++) v[c][(long)i * nr + r] = acc[(long)cls[i] * nr + r];
    }
    free(cls);
    free(acc);
    return 0;
}

double tno_masked_dot(int lat_level, int nr, int ncomp, const double* const* a, const double* const* b)
{
    const int nl = (1 << lat_level) + 1;
    uint8_t*  own = (uint8_t*)malloc((size_t)10 * nl * nl);
    tno_ownership(lat_level, own);
    double total = 0.0;
    for (int c = 0; c < ncomp; c++) {
        double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
        for (long i = 0; i < 10L * nl * nl; i++) {
            if (!own[i]) continue;
            for (int r = 0; r < nr; r++) s += a[c][i * nr + r] * b[c][i * nr + r];
        }
        total += s;
    }
    free(own);
    return total;
}

/* ========================================================================== */
/* Divergence / gradient (P1-iso-P2 / P1 coupling)                            */
/* ========================================================================== */

/* shape_coarse and its pieces (integrands.hpp:250-393). */
static double shape_rad_coarse(int cn, int frw, double z)
{
    if (cn / 3 == 0) return frw == 0 ? 0.25 * (3 - z) : 0.25 * (1 - z);
    return frw == 0 ? 0.25 * (1 + z) : 0.25 * (3 + z);
}
static double shape_lat_coarse(int cn, int flw, double xi, double eta)
{
    switch (cn % 3) {
    case 0:
        switch (flw) {
        case 0: return -0.5 * eta - 0.5 * xi + 1.0;
        case 1: return -0.5 * eta - 0.5 * xi + 0.5;
        case 2: return -0.5 * eta - 0.5 * xi + 0.5;
        default: return 0.5 * eta + 0.5 * xi;
        }
    case 1:
        switch (flw) {
        case 0: return 0.5 * xi;
        case 1: return 0.5 * xi + 0.5;
        case 2: return 0.5 * xi;
        default: return 0.5 - 0.5 * xi;
        }
    default:
        switch (flw) {
        case 0: return 0.5 * eta;
        case 1: return 0.5 * eta;
        case 2: return 0.5 * eta + 0.5;
        default: return 0.5 - 0.5 * eta;
        }
    }
}
static double shape_coarse(int cn, int frw, int flw, const double q[3])
{
    return shape_lat_coarse(cn, flw, q[0], q[1]) * shape_rad_coarse(cn, frw, q[2]);
}
/* fine_lateral_wedge_idx (kernel_helpers.hpp:600-608). */
static int fine_lat_wedge(int x, int y, int w)
{
    static const int idx[2][2][2] = {{{0, 1}, {2, 3}}, {{3, 2}, {1, 0}}};
    return idx[w][y % 2][x % 2];
}

/* B element matrix A[i][d*6+j] = -qw (J^-T grad_j)_d shape_coarse_i |det|
 * (divergence_kerngen.hpp:368-392). */
static void div_matrix(const tno_op* op, int d, int x, int y, int r, int w, double A[6][18])
{
    double ws[2][3][3], J[3][3], JiT[3][3];
    wedge_surface(op->coords, op->nl, d, x, y, ws);
    jacobian(ws[w], op->radii[r], op->radii[r + 1], QP, J);
    double det = fabs(det3(J));
    inv_transposed(J, det3(J), JiT);
    int frw = r % 2, flw = fine_lat_wedge(x, y, w);
    memset(A, 0, sizeof(double) * 108);
    for (int i = 0; i < 6; i++) {
        double si = shape_coarse(i, frw, flw, QP);
        for (int j = 0; j < 6; j++) {
            double gr[3], g[3];
            grad_shape(j, QP, gr);
            for (int a = 0; a < 3; a++) g[a] = JiT[a][0] * gr[0] + JiT[a][1] * gr[1] + JiT[a][2] * gr[2];
            for (int dd = 0; dd < 3; dd++) A[i][dd * 6 + j] += QW * (-g[dd] * si * det);
        }
    }
}

/* boundary treatment shared by B and B^T slow paths: returns a rotation per
 * wedge (node-wise ordering) for free-slip and a column mask (Dirichlet). */
static int bt_boundary(const tno_op* op, int d, int x, int y, int r, double R[2][324], double colmask[18], int* node_wise)
{
    int at_cmb = (r == 0), at_surface = (r + 1 == op->nr - 1);
    for (int i = 0; i < 18; i++) colmask[i] = 1.0;
    *node_wise = 0;
    if (!(at_cmb || at_surface)) return 0;
    int bcf = at_cmb ? op->bc_cmb : op->bc_surface;
    if (bcf == 1) {
        for (int dd = 0; dd < 3; dd++)
            for (int j = 0; j < 6; j++)
                if ((at_cmb && j < 3) || (at_surface && j >= 3)) colmask[dd * 6 + j] = 0.0;
    } else if (bcf == 2) {
        static const int ox[2][3] = {{0, 1, 0}, {1, 0, 1}}, oy[2][3] = {{0, 0, 1}, {1, 1, 0}};
        *node_wise = 1;
        for (int w = 0; w < 2; w++) {
            memset(R[w], 0, sizeof(double) * 324);
            for (int i = 0; i < 18; i++) R[w][i * 18 + i] = 1.0;
            for (int b = 0; b < 3; b++) {
                double nrm[3], Ri[3][3];
                physical_coords(op, d, x + ox[w][b], y + oy[w][b], r + (at_cmb ? 0 : 1), nrm);
                trafo_nt(nrm, Ri);
                int off = at_cmb ? 0 : 9;
                for (int a = 0; a < 3; a++)
                    for (int c = 0; c < 3; c++) R[w][(off + b * 3 + a) * 18 + off + b * 3 + c] = Ri[a][c];
            }
        }
        int ns = at_surface ? 3 : 0, ne = at_surface ? 6 : 3;
        for (int nn = ns; nn < ne; nn++) colmask[nn * 3] = 0.0; /* node-wise index of the normal component */
    }
    return 1;
}

int tno_divergence(const tno_op* op, const double* const* u, double* p)
{
    const int nl = op->nl, nr = op->nr, nlc = (nl + 1) / 2, nrc = (nr + 1) / 2;
    memset(p, 0, sizeof(double) * 10L * nlc * nlc * nrc);
    /* coarse nodes receive from four fine x-cells; sweep x mod 4 classes */
    for (int phase = 0; phase < 4; phase++) {
#pragma omp parallel for collapse(2) schedule(static)
        for (int d = 0; d < 10; d++)
            for (int xq = 0; xq < (nl - 1 + 3 - phase) / 4; xq++) {
                int x = 4 * xq + phase;
                for (int y = 0; y < nl - 1; y++)
                    for (int r = 0; r < nr - 1; r++) {
                        double R[2][324], colmask[18];
                        int    nw;
                        bt_boundary(op, d, x, y, r, R, colmask, &nw);
                        for (int w = 0; w < 2; w++) {
                            double A[6][18], s[18], out[6];
                            div_matrix(op, d, x, y, r, w, A);
                            for (int dd = 0; dd < 3; dd++)
                                for (int n = 0; n < 6; n++)
                                    s[dd * 6 + n] = u[dd][IDX4(nl, nr, d, x + WOFF[w][n][0], y + WOFF[w][n][1], r + WOFF[w][n][2])];
                            if (nw) {
                                double At[6][18], sn[18], sr[18];
                                for (int i = 0; i < 6; i++)
                                    for (int dj = 0; dj < 3; dj++)
                                        for (int j = 0; j < 6; j++) At[i][j * 3 + dj] = A[i][j + dj * 6];
                                for (int dd = 0; dd < 3; dd++)
                                    for (int n = 0; n < 6; n++) sn[n * 3 + dd] = s[n + dd * 6];
                                /* A = At R^T, s = R s */
                                for (int i = 0; i < 6; i++)
                                    for (int j = 0; j < 18; j++) {
                                        double acc = 0;
                                        for (int k = 0; k < 18; k++) acc += At[i][k] * R[w][j * 18 + k];
                                        A[i][j] = acc;
                                    }
                                for (int i = 0; i < 18; i++) {
                                    double acc = 0;
                                    for (int k = 0; k < 18; k++) acc += R[w][i * 18 + k] * sn[k];
                                    sr[i] = acc;
                                }
                                memcpy(s, sr, sizeof(sr));
                            }
                            for (int i = 0; i < 6; i++) {
                                double acc = 0;
                                for (int j = 0; j < 18; j++) acc += A[i][j] * colmask[j] * s[j];
                                out[i] = acc;
                            }
                            for (int i = 0; i < 6; i++)
                                p[IDX4(nlc, nrc, d, x / 2 + WOFF[w][i][0], y / 2 + WOFF[w][i][1], r / 2 + WOFF[w][i][2])] += out[i];
                        }
                    }
            }
    }
    return 0;
}

int tno_gradient(const tno_op* op, const double* p, double* const* u)
{
    const int nl = op->nl, nr = op->nr, nlc = (nl + 1) / 2, nrc = (nr + 1) / 2;
    zero_vec(u, 3, 10L * nl * nl * nr);
    CELL_LOOP_BEGIN(nl, nr)
    double R[2][324], rowmask[18];
    int    nw;
    bt_boundary(op, d, x, y, r, R, rowmask, &nw);
    for (int w = 0; w < 2; w++) {
        double A[6][18], pc[6], out[18];
        div_matrix(op, d, x, y, r, w, A); /* B^T element = transpose of B element */
        for (int j = 0; j < 6; j++)
            pc[j] = p[IDX4(nlc, nrc, d, x / 2 + WOFF[w][j][0], y / 2 + WOFF[w][j][1], r / 2 + WOFF[w][j][2])];
        for (int i = 0; i < 18; i++) {
            double acc = 0;
            for (int j = 0; j < 6; j++) acc += A[j][i] * pc[j];
            out[i] = acc;
        }
        if (nw) {
            double on[18], rot[18];
            for (int dd = 0; dd < 3; dd++)
                for (int n = 0; n < 6; n++) on[n * 3 + dd] = out[n + dd * 6];
            for (int i = 0; i < 18; i++) {
                double acc = 0;
                for (int k = 0; k < 18; k++) acc += R[w][i * 18 + k] * on[k];
                rot[i] = acc * rowmask[i];
            }
            for (int i = 0; i < 18; i++) {
                double acc = 0;
                for (int k = 0; k < 18; k++) acc += R[w][k * 18 + i] * rot[k];
                on[i] = acc;
            }
            for (int dd = 0; dd < 3; dd++)
                for (int n = 0; n < 6; n++) out[n + dd * 6] = on[n * 3 + dd];
        } else
            for (int i = 0; i < 18; i++) out[i] *= rowmask[i];
        for (int dd = 0; dd < 3; dd++)
            for (int n = 0; n < 6; n++)
                u[dd][IDX4(nl, nr, d, x + WOFF[w][n][0], y + WOFF[w][n][1], r + WOFF[w][n][2])] += out[dd * 6 + n];
    }
    CELL_LOOP_END
    return 0;
}

/* ========================================================================== */
/* Mass matrices                                                              */
/* ========================================================================== */

/* Felippa 3x2 rule (quadrature.hpp:57-100). */
static const double QP6[6][3] = {{0.6666666666666666, 0.1666666666666667, -0.5773502691896257},
                                 {0.1666666666666667, 0.6666666666666666, -0.5773502691896257},
                                 {0.1666666666666667, 0.1666666666666667, -0.5773502691896257},
                                 {0.6666666666666666, 0.1666666666666667, 0.5773502691896257},
                                 {0.1666666666666667, 0.6666666666666666, 0.5773502691896257},
                                 {0.1666666666666667, 0.1666666666666667, 0.5773502691896257}};
static const double QW6 = 0.1666666666666667;

static void mass_matrix(int nl, const double* coords, const double* radii, int d, int x, int y, int r, int w,
                        const double* kloc, double A[6][6])
{
    double ws[2][3][3];
    wedge_surface(coords, nl, d, x, y, ws);
    double r1 = radii[r], r2 = radii[r + 1], grad_r = 0.5 * (r2 - r1);
    memset(A, 0, sizeof(double) * 36);
    for (int q = 0; q < 6; q++) {
        double col[3][3];
        for (int i = 0; i < 3; i++) {
            col[0][i] = ws[w][1][i] - ws[w][0][i];
            col[1][i] = ws[w][2][i] - ws[w][0][i];
            col[2][i] = (1 - QP6[q][0] - QP6[q][1]) * ws[w][0][i] + QP6[q][0] * ws[w][1][i] + QP6[q][1] * ws[w][2][i];
        }
        double Jl[3][3];
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) Jl[i][j] = col[j][i];
        double dl   = fabs(det3(Jl));
        double rq   = r1 + 0.5 * (r2 - r1) * (1 + QP6[q][2]);
        double keval = 1.0;
        if (kloc) {
            keval = 0.0;
            for (int j = 0; j < 6; j++) keval += shape(j, QP6[q]) * kloc[j];
        }
        for (int i = 0; i < 6; i++)
            for (int j = 0; j < 6; j++) {
                double si = shape_lat(i, QP6[q][0], QP6[q][1]) * shape_rad(i, QP6[q][2]);
                double sj = shape_lat(j, QP6[q][0], QP6[q][1]) * shape_rad(j, QP6[q][2]);
                A[i][j] += QW6 * keval * (si * sj * rq * rq * grad_r * dl);
            }
    }
}

int tno_kmass_lumped(int nl, int nr, const double* coords, const double* radii, const double* k, double* diag)
{
    memset(diag, 0, sizeof(double) * 10L * nl * nl * nr);
    CELL_LOOP_BEGIN(nl, nr)
    for (int w = 0; w < 2; w++) {
        double kl[6], A[6][6];
        for (int n = 0; n < 6; n++) kl[n] = k[IDX4(nl, nr, d, x + WOFF[w][n][0], y + WOFF[w][n][1], r + WOFF[w][n][2])];
        mass_matrix(nl, coords, radii, d, x, y, r, w, kl, A);
        for (int i = 0; i < 6; i++) {
            double rs = 0;
            for (int j = 0; j < 6; j++) rs += A[i][j];
            diag[IDX4(nl, nr, d, x + WOFF[w][i][0], y + WOFF[w][i][1], r + WOFF[w][i][2])] += rs;
        }
    }
    CELL_LOOP_END
    return 0;
}

int tno_vector_mass(int nl, int nr, const double* coords, const double* radii, const double* const* src,
                    double* const* dst)
{
    zero_vec(dst, 3, 10L * nl * nl * nr);
    CELL_LOOP_BEGIN(nl, nr)
    for (int w = 0; w < 2; w++) {
        double A[6][6];
        mass_matrix(nl, coords, radii, d, x, y, r, w, NULL, A);
        for (int c = 0; c < 3; c++) {
            double s[6];
            for (int n = 0; n < 6; n++) s[n] = src[c][IDX4(nl, nr, d, x + WOFF[w][n][0], y + WOFF[w][n][1], r + WOFF[w][n][2])];
            for (int i = 0; i < 6; i++) {
                double acc = 0;
                for (int j = 0; j < 6; j++) acc += A[i][j] * s[j];
                dst[c][IDX4(nl, nr, d, x + WOFF[w][i][0], y + WOFF[w][i][1], r + WOFF[w][i][2])] += acc;
            }
        }
    }
    CELL_LOOP_END
    return 0;
}

/* ========================================================================== */
/* Transfers                                                                  */
/* ========================================================================== */

/* prolongation_constant_weight (fe/wedge/shell/grid_transfer_constant.hpp:24-89). */
static double pweight(int xf, int yf, int rf, int xc, int yc, int rc)
{
    int dx = xf - 2 * xc, dy = yf - 2 * yc, dr = rf - 2 * rc;
    double lat = 0.0;
    if (dx == 0 && dy == 0) lat = 1.0;
    else if (dy == 0 && (dx == 1 || dx == -1)) lat = 0.5;
    else if (dx == 0 && (dy == 1 || dy == -1)) lat = 0.5;
    else if (dx == -1 && dy == 1) lat = 0.5;
    else if (dx == 1 && dy == -1) lat = 0.5;
    if (dr == 0) return lat;
    if (dr == 1 || dr == -1) return 0.5 * lat;
    return 0.0;
}
static const int POFF[7][2] = {{-1, 0}, {-1, 1}, {0, 1}, {1, 0}, {1, -1}, {0, -1}, {0, 0}};

int tno_prolongate_add(int llf, int rlf, int ncomp, const double* const* coarse, double* const* fine)
{
    const int nlf = (1 << llf) + 1, nrf = (1 << rlf) + 1, nlc = (nlf + 1) / 2, nrc = (nrf + 1) / 2;
    /* gather form per fine node of the additive scatter in prolongation_constant.hpp:166-190 */
#pragma omp parallel for collapse(2) schedule(static)
    for (int d = 0; d < 10; d++)
        for (int x = 0; x < nlf; x++)
            for (int y = 0; y < nlf; y++)
                for (int r = 0; r < nrf; r++)
                    for (int c = 0; c < ncomp; c++) {
                        double acc = 0.0;
                        for (int xc = (x - 1) / 2 < 0 ? 0 : (x - 1) / 2; xc <= (x + 1) / 2 && xc < nlc; xc++)
                            for (int yc = (y - 1) / 2 < 0 ? 0 : (y - 1) / 2; yc <= (y + 1) / 2 && yc < nlc; yc++)
                                for (int rc = (r - 1) / 2 < 0 ? 0 : (r - 1) / 2; rc <= (r + 1) / 2 && rc < nrc; rc++) {
                                    int dx = x - 2 * xc, dy = y - 2 * yc, dr = r - 2 * rc, in = 0;
                                    for (int o = 0; o < 7; o++)
                                        if (POFF[o][0] == dx && POFF[o][1] == dy) in = 1;
                                    if (!in || dr < -1 || dr > 1) continue;
                                    acc += pweight(x, y, r, xc, yc, rc) * coarse[c][IDX4(nlc, nrc, d, xc, yc, rc)];
                                }
                        fine[c][IDX4(nlf, nrf, d, x, y, r)] += acc;
                    }
    return 0;
}

int tno_restrict(int llf, int rlf, int ncomp, const double* const* fine, double* const* coarse)
{
    const int nlf = (1 << llf) + 1, nrf = (1 << rlf) + 1, nlc = (nlf + 1) / 2, nrc = (nrf + 1) / 2;
    uint8_t*  own = (uint8_t*)malloc((size_t)10 * nlf * nlf);
    tno_ownership(llf, own);
#pragma omp parallel for collapse(2) schedule(static)
    for (int d = 0; d < 10; d++)
        for (int xc = 0; xc < nlc; xc++)
            for (int yc = 0; yc < nlc; yc++)
                for (int rc = 0; rc < nrc; rc++)
                    for (int c = 0; c < ncomp; c++) {
                        double acc = 0.0;
                        for (int rr = -1; rr <= 1; rr++)
                            for (int o = 0; o < 7; o++) {
                                int xf = 2 * xc + POFF[o][0], yf = 2 * yc + POFF[o][1], rf = 2 * rc + rr;
                                if (xf < 0 || xf >= nlf || yf < 0 || yf >= nlf || rf < 0 || rf >= nrf) continue;
                                if (!own[LAT(nlf, d, xf, yf)]) continue;
                                acc += pweight(xf, yf, rf, xc, yc, rc) * fine[c][IDX4(nlf, nrf, d, xf, yf, rf)];
                            }
                        coarse[c][IDX4(nlc, nrc, d, xc, yc, rc)] = acc;
                    }
    free(own);
    tno_interface_sum(llf - 1, nrc, ncomp, coarse);
    return 0;
}

/* ========================================================================== */
/* GCA two-grid coarsening                                                    */
/* ========================================================================== */

int tno_gca_coarsen(const tno_op* fine_op, const double* fine_mats, double* coarse_mats)
{
    return tno_gca_coarsen_w(fine_op, fine_mats, NULL, coarse_mats);
}

/* linw: per fine node the two linear-transfer weights (InterpolationMode::Linear, gca.hpp:231-243, :327-342),
 * or NULL for the constant mode. */
int tno_gca_coarsen_w(const tno_op* fine_op, const double* fine_mats, const double* linw, double* coarse_mats)
{
    const int nlf = fine_op->nl, nrf = fine_op->nr, nlc = (nlf + 1) / 2, nrc = (nrf + 1) / 2;
    static const int shifts[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {1, 1, 0}, {0, 0, 1}, {1, 0, 1}, {0, 1, 1}, {1, 1, 1}};
#pragma omp parallel for collapse(2) schedule(static)
    for (int d = 0; d < 10; d++)
        for (int xc = 0; xc < nlc - 1; xc++)
            for (int yc = 0; yc < nlc - 1; yc++)
                for (int rc = 0; rc < nrc - 1; rc++) {
                    double Ac[2][324];
                    memset(Ac, 0, sizeof(Ac));
                    for (int h = 0; h < 8; h++) {
                        int fx = 2 * xc + shifts[h][0], fy = 2 * yc + shifts[h][1], fr = 2 * rc + shifts[h][2];
                        for (int w = 0; w < 2; w++) {
                            double P[6][6], Af[324], PV[324], T[324];
                            memset(P, 0, sizeof(P));
                            /* gca.hpp:204-383 (constant interpolation mode) */
                            for (int fl = 0; fl < 6; fl++) {
                                int ix = fx + WOFF[w][fl][0], iy = fy + WOFF[w][fl][1], ir = fr + WOFF[w][fl][2];
                                if (ix % 2 == 0 && iy % 2 == 0 && ir % 2 == 0) {
                                    P[fl][fl] = 1.0;
                                    continue;
                                }
                                int rb = ir < nrf - 1 ? ir / 2 : ir / 2 - 1, rt = rb + 1;
                                double lw0 = 0.5, lw1 = 0.5;
                                if (linw) {
                                    long fi = IDX4(nlf, nrf, d, ix, iy, ir);
                                    lw0 = linw[2 * fi];
                                    lw1 = linw[2 * fi + 1];
                                }
                                if (ix % 2 == 0 && iy % 2 == 0) {
                                    if (fl == 2 || fl == 5) { P[fl][2] = lw0; P[fl][5] = lw1; }
                                    else if (fl == 0 || fl == 3) { P[fl][0] = lw0; P[fl][3] = lw1; }
                                    else { P[fl][1] = lw0; P[fl][4] = lw1; }
                                    continue;
                                }
                                int x0, x1, y0, y1, cl[4];
                                if (ix % 2 == 0) {
                                    x0 = ix / 2; x1 = ix / 2; y0 = iy / 2; y1 = iy / 2 + 1;
                                    cl[0] = 0; cl[1] = 2; cl[2] = 3; cl[3] = 5;
                                } else if (iy % 2 == 0) {
                                    x0 = ix / 2; x1 = ix / 2 + 1; y0 = iy / 2; y1 = iy / 2;
                                    cl[0] = 0; cl[1] = 1; cl[2] = 3; cl[3] = 4;
                                } else {
                                    x0 = ix / 2 + 1; x1 = ix / 2; y0 = iy / 2; y1 = iy / 2 + 1;
                                    cl[0] = 1; cl[1] = 2; cl[2] = 4; cl[3] = 5;
                                }
                                if (linw) {
                                    P[fl][cl[0]] = lw0;
                                    P[fl][cl[1]] = lw0;
                                    P[fl][cl[2]] = lw1;
                                    P[fl][cl[3]] = lw1;
                                    continue;
                                }
                                P[fl][cl[0]] = pweight(ix, iy, ir, x0, y0, rb);
                                P[fl][cl[1]] = pweight(ix, iy, ir, x1, y1, rb);
                                P[fl][cl[2]] = pweight(ix, iy, ir, x0, y0, rt);
                                P[fl][cl[3]] = pweight(ix, iy, ir, x1, y1, rt);
                            }
                            if (fine_mats) {
                                long c = IDX4(nlf - 1, nrf - 1, d, fx, fy, fr);
                                memcpy(Af, fine_mats + (c * 2 + w) * 324, sizeof(Af));
                            } else
                                local_matrix(fine_op, d, fx, fy, fr, w, Af);
                            memset(PV, 0, sizeof(PV));
                            for (int dd = 0; dd < 3; dd++)
                                for (int i = 0; i < 6; i++)
                                    for (int j = 0; j < 6; j++) PV[(i + dd * 6) * 18 + j + dd * 6] = P[i][j];
                            /* T = Af PV ; PTAP = PV^T T */
                            for (int i = 0; i < 18; i++)
                                for (int j = 0; j < 18; j++) {
                                    double acc = 0;
                                    for (int k = 0; k < 18; k++) acc += Af[i * 18 + k] * PV[k * 18 + j];
                                    T[i * 18 + j] = acc;
                                }
                            int target;
                            if ((w == 0 && (h == 0 || h == 1 || h == 2 || h == 4 || h == 5 || h == 6)) ||
                                (w == 1 && (h == 0 || h == 4)))
                                target = 0;
                            else
                                target = 1;
                            for (int i = 0; i < 18; i++)
                                for (int j = 0; j < 18; j++) {
                                    double acc = 0;
                                    for (int k = 0; k < 18; k++) acc += PV[k * 18 + i] * T[k * 18 + j];
                                    Ac[target][i * 18 + j] += acc;
                                }
                        }
                    }
                    long c = IDX4(nlc - 1, nrc - 1, d, xc, yc, rc);
                    memcpy(coarse_mats + (c * 2 + 0) * 324, Ac[0], sizeof(double) * 324);
                    memcpy(coarse_mats + (c * 2 + 1) * 324, Ac[1], sizeof(double) * 324);
                }
    return 0;
}

/* ========================================================================== */
/* Adjoint: derivative of lambda^T A u with respect to log(eta_cell)          */
/* ========================================================================== */

/* g_cell += lambda^T (dA / dlog eta_cell) u for the Q0 coefficient. A is
 * linear in eta_cell, so the derivative is the cell's own masked wedge
 * matrices (slow-path Dirichlet masks, epsilon_divdiv_kerngen.hpp:1101-1124)
 * evaluated at eta_cell. Free-slip boundaries are not supported here. */
int tno_epsdivdiv_vjp_logeta(const tno_op* op, const double* const* u, const double* const* lam, double* g)
{
    if (!op->k_q0) return -1;
    const int nl = op->nl, nr = op->nr;
#pragma omp parallel for collapse(2) schedule(static)
    for (int d = 0; d < 10; d++)
        for (int x = 0; x < nl - 1; x++)
            for (int y = 0; y < nl - 1; y++)
                for (int r = 0; r < nr - 1; r++) {
                    /* A is linear in eta_cell: d(lambda^T A u)/d log eta_cell is the
                     * cell's own contribution lambda_e^T A_e(eta_cell) u_e, boundary
                     * treatment included (slow path). */
                    double A[2][324], outw[2][18];
                    local_matrix(op, d, x, y, r, 0, A[0]);
                    local_matrix(op, d, x, y, r, 1, A[1]);
                    slow_cell_local(op, d, x, y, r, A, u, outw);
                    double acc = 0.0;
                    for (int w = 0; w < 2; w++)
                        for (int dim = 0; dim < 3; dim++)
                            for (int n = 0; n < 6; n++)
                                acc += lam[dim][IDX4(nl, nr, d, x + WOFF[w][n][0], y + WOFF[w][n][1],
                                                     r + WOFF[w][n][2])] *
                                       outw[w][dim * 6 + n];
                    g[IDX4(nl - 1, nr - 1, d, x, y, r)] += acc;
                }
    return 0;
}
