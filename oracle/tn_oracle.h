/* CPU oracle for the TERRA-NG Stokes hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * This library restates, in plain C and FP64, the reference's algorithms for
 * the thick-shell mesh and the Stokes operators so that the CUDA product can be
 * checked against it. Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load it; the product never links or calls it.
 *
 * Layout: nodal arrays (10, nl, nl, nr) with r fastest; lateral coordinates
 * (10, nl, nl, 3); radii (nr). Cell arrays (10, nl-1, nl-1, nr-1).
 * Boundary conditions: 0 Neumann, 1 Dirichlet, 2 free-slip (grid/shell/bit_masks.hpp:20-25).
 */
#ifndef TN_ORACLE_H
#define TN_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- mesh ---------------------------------------------------------------- */
int  tno_unit_sphere_coords(int lat_level, double* out);
int  tno_uniform_radii(double r_min, double r_max, int num_shells, double* out);
/* class id per lateral node (10, nl, nl); -1 for nodes held by one diamond only.
 * Returns the number of classes or a negative value on error. */
int  tno_duplicate_classes(int lat_level, int32_t* class_of_lat);
/* ownership per lateral node (10, nl, nl): 1 for the copy in the lowest diamond. */
int  tno_ownership(int lat_level, uint8_t* owned_lat);
/* boundary flag per node (10, nl, nl, nr) (grid/shell/bit_masks.hpp:82-136). */
int  tno_boundary_mask(int nl, int nr, uint8_t* mask);

/* ---- operators ------------------------------------------------------------
 * All applies write dst in Replace mode and do NOT sum interface duplicates;
 * call tno_interface_sum afterwards for the CommunicateAdditively result.   */
typedef struct {
    int           nl, nr;
    const double* coords;  /* (10, nl, nl, 3) */
    const double* radii;   /* (nr) */
    const double* k;       /* nodal coefficient (10, nl, nl, nr), or NULL when k_q0 is set */
    const double* k_q0;    /* per-cell coefficient (10, nl-1, nl-1, nr-1), or NULL */
    int           bc_cmb, bc_surface;
    int           diagonal;
} tno_op;

/* epsilon-div-div, reference slow path: assembled 18x18 wedge matrices with
 * boundary masks / free-slip rotation (epsilon_divdiv_kerngen.hpp:1013-1242, 2315-2392). */
int tno_epsdivdiv_slow(const tno_op* op, const double* const* src, double* const* dst);
/* epsilon-div-div, reference fast paths (Dirichlet/Neumann :1245-1607, free-slip :1638-2198). */
int tno_epsdivdiv_fast(const tno_op* op, const double* const* src, double* const* dst);
/* one wedge-local 18x18 matrix, unmasked (assemble_local_matrix, :2315-2392). */
int tno_epsdivdiv_local_matrix(const tno_op* op, int d, int x, int y, int r, int wedge, double* A18x18);
/* stored-matrix (GCA) apply: mats (10, nl-1, nl-1, nr-1, 2, 18, 18) row-major, slow-path masks. */
int tno_epsdivdiv_stored(const tno_op* op, const double* mats, const double* const* src, double* const* dst);

/* divergence B: velocity on (nl, nr) -> pressure on coarse ((nl+1)/2, (nr+1)/2)
 * (divergence_kerngen.hpp:341-466); gradient B^T (gradient_kerngen.hpp:338-500). */
int tno_divergence(const tno_op* op, const double* const* u, double* p_coarse);
int tno_gradient(const tno_op* op, const double* p_coarse, double* const* u);

/* lumped k-weighted pressure mass diagonal (kmass.hpp:98-181 with lumping). */
int tno_kmass_lumped(int nl, int nr, const double* coords, const double* radii, const double* k, double* diag);
/* vector mass apply, 6-point rule (vector_mass.hpp:60-150). */
int tno_vector_mass(int nl, int nr, const double* coords, const double* radii, const double* const* src,
                    double* const* dst);

/* interface sum: every duplicated node receives the sum over its class (SUM
 * reduction of communication_plan.hpp:48-71). ncomp arrays of shape (10,nl,nl,nr). */
int tno_interface_sum(int lat_level, int nr, int ncomp, double* const* v);

/* constant-weight transfers (prolongation_constant.hpp:146-191, restriction_constant.hpp:133-250).
 * Prolongation is additive (dst += P src); restriction is Replace, ownership-masked,
 * and includes the interface sum. Levels are the fine lateral/radial levels. */
int tno_prolongate_add(int lat_level_f, int rad_level_f, int ncomp, const double* const* coarse, double* const* fine);
int tno_restrict(int lat_level_f, int rad_level_f, int ncomp, const double* const* fine, double* const* coarse);

/* GCA two-grid coarsening (gca.hpp:154-530): fine_mats == NULL means the fine
 * operator's on-the-fly local matrices from `fine_op` (Neumann) are used. Output
 * (10, nlc-1, nlc-1, nrc-1, 2, 18, 18). */
int tno_gca_coarsen(const tno_op* fine_op, const double* fine_mats, double* coarse_mats);
int tno_gca_coarsen_w(const tno_op* fine_op, const double* fine_mats, const double* linw, double* coarse_mats);

/* owned-masked dot of ncomp-component nodal vectors. */
double tno_masked_dot(int lat_level, int nr, int ncomp, const double* const* a, const double* const* b);

/* adjoint / VJP with respect to per-cell log-viscosity for the Q0 coefficient:
 * g_cell += lambda^T dA/dlog(eta_cell) u = lambda_e^T A_e(eta_cell) u_e, with
 * the operator's slow-path boundary handling (Neumann, Dirichlet, free-slip). */
int tno_epsdivdiv_vjp_logeta(const tno_op* op, const double* const* u, const double* const* lam, double* g_cell);

int tno_set_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
