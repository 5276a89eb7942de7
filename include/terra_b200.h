/*
 * terra_b200 -- C ABI of the B200-native TERRA-NG Stokes hot path.
 *
 * Every entry point is extern "C", takes plain pointers and sizes, and returns
 * an int status (TN_OK == 0, negative on error; tn_last_error() describes the
 * last failure of the calling thread). Array arguments named *_dev are device
 * pointers aligned to their element size. Input arrays are staged into shared
 * memory by bulk copies of whole 16-byte blocks, so the 16-byte-aligned blocks
 * that contain an input array must be readable device memory (true for any
 * array inside a cudaMalloc / torch allocation).
 * Operations run asynchronously on the caller's CUDA stream (NULL = legacy
 * default stream) unless documented as synchronous. An object lives on the
 * device that was current when it was created, and that device must be the
 * current one whenever the object (or anything built on it) is used.
 *
 * Data layout is the reference's diamond-grid layout (src/terra/grid/
 * grid_types.hpp:12-113, Kokkos::LayoutRight): a nodal scalar field is
 * (10, nl, nl, nr) with r fastest; a velocity field is three such arrays (the
 * SoA Grid4DDataVec); lateral coordinates are (10, nl, nl, 3); cell fields
 * are (10, nl-1, nl-1, nr-1). Level indices count from 0 (coarsest).
 *
 * Each declaration names the reference interface it replaces (paths inside the
 * reference project).
 */
#ifndef TERRA_B200_H
#define TERRA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status, enums -------------------------------------------------------- */
enum {
    TN_OK               = 0,
    TN_ERR_ARG          = -1, /* invalid argument (extent mismatch, bad pointer, ...) */
    TN_ERR_CUDA         = -2, /* CUDA runtime error */
    TN_ERR_ALLOC        = -3, /* device allocation failed */
    TN_ERR_STATE        = -4, /* object not in a state that allows the call */
    TN_ERR_DEVICE       = -5, /* a kernel reported a device-side error (bounded wait expired) */
    TN_ERR_UNSUPPORTED  = -6, /* option combination not implemented */
    TN_ERR_NOT_CONVERGED = -7 /* iterative solve stopped before reaching its tolerance */
};
enum { TN_F64 = 0, TN_F32 = 1 };
/* BoundaryConditionFlag (src/terra/grid/shell/bit_masks.hpp:20-25) */
enum { TN_NEUMANN = 0, TN_DIRICHLET = 1, TN_FREESLIP = 2 };
/* OperatorApplyMode / OperatorCommunicationMode (src/terra/linalg/operator.hpp:29-51) */
enum { TN_REPLACE = 0, TN_ADD = 1 };
enum { TN_SKIP_COMMUNICATION = 0, TN_COMMUNICATE_ADDITIVELY = 1 };

/* OperatorStoredMatrixMode (src/terra/linalg/operator.hpp:29-51); Selective is not provided */
enum { TN_STORED_OFF = 0, TN_STORED_FULL = 1 };

typedef struct tn_shell    tn_shell;
typedef struct tn_operator tn_operator;
typedef struct tn_solver   tn_solver;

/* Message of the last failed call on this thread ("" if none). */
const char* tn_last_error(void);
/* Library version string. */
const char* tn_version(void);
/* Kernel launches issued by this library since it was loaded (launch calls on
 * any stream; for counting the device work of a call). */
uint64_t tn_kernel_launch_count(void);

/* ---- mesh hierarchy --------------------------------------------------------
 * Replaces DistributedDomain / DomainInfo with one subdomain per diamond plus
 * subdomain_unit_sphere_single_shell_coords, subdomain_shell_radii and the
 * boundary / ownership masks (src/terra/grid/shell/spherical_shell.hpp:825-2967,
 * src/terra/grid/shell/bit_masks.hpp:82-136, src/terra/grid/bit_masks.hpp:27-85).
 * Builds num_levels levels; level num_levels-1 has lateral refinement
 * lat_level and radial refinement rad_level (2^rad_level layers), each coarser
 * level halves both. Uniform radii in [r_min, r_max]. Synchronous.          */
int tn_shell_create(int lat_level, int rad_level, int num_levels, double r_min, double r_max, tn_shell** out);
void tn_shell_destroy(tn_shell* shell);
int tn_shell_num_levels(const tn_shell* shell, int* num_levels);
int tn_shell_level_dims(const tn_shell* shell, int level, int* nl, int* nr);
/* Host copies (synchronous). coords (10,nl,nl,3); radii (nr); ownership and
 * boundary mask (10,nl,nl,nr) as uint8 flags (NodeOwnershipFlag,
 * ShellBoundaryFlag values); class_of_lat (10,nl,nl): duplicate-node class or -1. */
int tn_shell_copy_coords(const tn_shell* shell, int level, double* coords_host);
int tn_shell_copy_radii(const tn_shell* shell, int level, double* radii_host);
int tn_shell_copy_ownership(const tn_shell* shell, int level, uint8_t* owned_host);
int tn_shell_copy_boundary_mask(const tn_shell* shell, int level, uint8_t* mask_host);
int tn_shell_duplicate_classes(const tn_shell* shell, int level, int32_t* class_of_lat_host, int* num_classes);
/* Host-only mesh generation of one level (no device needed): the same
 * generator tn_shell_create uses. Any output pointer may be NULL. Shapes:
 * coords (10,nl,nl,3), radii (nr), owned (10,nl,nl), class_of_lat (10,nl,nl). */
int tn_mesh_generate_host(int lat_level, int rad_level, double r_min, double r_max, double* coords_host,
                          double* radii_host, uint8_t* owned_lat_host, int32_t* class_of_lat_host, int* num_classes);
/* Device error word written by bounded waits inside kernels (0 = none);
 * reading it synchronizes the device and clears it. */
int tn_shell_check_device_error(tn_shell* shell, int* code);

/* ---- epsilon-div-div operator ----------------------------------------------
 * Replaces EpsilonDivDivKerngen<ScalarT> (src/terra/fe/wedge/operators/shell/
 * epsilon_divdiv_kerngen.hpp:205-216 constructor, :447-528 setters, :577-792
 * apply_impl). Exactly one of k_nodal_dev (10,nl,nl,nr) or k_cell_dev
 * (10,nl-1,nl-1,nr-1; set_q0_coefficient_field) is non-NULL; it is copied.
 * Arrays are in the operator's precision (TN_F64 / TN_F32). Defaults:
 * Replace + CommunicateAdditively. Requires a level with at least 2 layers. */
int tn_epsdivdiv_create(tn_shell* shell, int level, int precision, const void* k_nodal_dev, const void* k_cell_dev,
                        int bc_cmb, int bc_surface, int diagonal, tn_operator** out);
void tn_operator_destroy(tn_operator* op);
/* Coupling blocks of the P1-iso-P2 / P1 pair between velocity_level and the
 * pressure level velocity_level-1:
 *   divergence B  (DivergenceKerngen, src/terra/fe/wedge/operators/shell/
 *                  divergence_kerngen.hpp:125-257): src 3 velocity comps, dst 1 pressure;
 *   gradient  B^T (GradientKerngen, gradient_kerngen.hpp:125-259): src 1, dst 3;
 *   Stokes [A B^T; B 0] (EpsDivDivStokes, epsilon_divdiv_stokes.hpp:39-84):
 *                  src / dst 4 components (u_x, u_y, u_z, p), Replace mode only. */
int tn_divergence_create(tn_shell* shell, int velocity_level, int precision, int bc_cmb, int bc_surface,
                         tn_operator** out);
int tn_gradient_create(tn_shell* shell, int velocity_level, int precision, int bc_cmb, int bc_surface,
                       tn_operator** out);
int tn_stokes_create(tn_shell* shell, int velocity_level, int precision, const void* k_nodal_dev,
                     const void* k_cell_dev, int bc_cmb, int bc_surface, tn_operator** out);
/* Number of source / destination component pointers an apply takes. */
int tn_operator_components(const tn_operator* op, int* src_components, int* dst_components);
/* set_operator_apply_and_communication_modes (epsilon_divdiv_kerngen.hpp:447-453) */
int tn_operator_set_modes(tn_operator* op, int apply_mode, int comm_mode);
/* set_diagonal (epsilon_divdiv_kerngen.hpp:455) */
int tn_operator_set_diagonal(tn_operator* op, int diagonal);
/* set_boundary_conditions (epsilon_divdiv_kerngen.hpp:474-481). With free slip
 * on both boundaries an epsilon-div-div operator adds the reference's null-space
 * penalty dst += 1e-7 sum_i (n_i^T src)_owned n_i over the three orthonormal
 * rotation modes n_i, on every interface copy before the interface sum and not
 * in diagonal mode (init_penalty and apply_impl, epsilon_divdiv_kerngen.hpp:
 * 324-445, :711-785); the modes are built by the first apply or this call
 * (synchronous, before any stream capture). */
int tn_operator_set_boundary_conditions(tn_operator* op, int bc_cmb, int bc_surface);
/* Override the CTA tile (0 = default); for tuning. */
int tn_operator_set_tile(tn_operator* op, int tile_y, int chunk_x);
/* apply_impl: dst = A src (Replace) or dst += A src (Add); with
 * CommunicateAdditively the interface duplicates of dst are summed afterwards.
 * src and dst are arrays of device pointers, one per component
 * (tn_operator_components). */
int tn_operator_apply(tn_operator* op, const void* const* src_dev, void* const* dst_dev, void* stream);

/* Backward of tn_operator_apply for an epsilon-div-div operator with a
 * per-cell (Q0) coefficient (no counterpart in the reference, which has no
 * adjoint): grad_logeta_cell_dev[e] = d(lambda^T A u)/d log(eta_e) =
 * lambda_e^T A_e(eta_e) u_e, boundary treatment included, written (not
 * accumulated); when grad_u_dev is not NULL also grad_u = A^T lambda = A lambda
 * (A is symmetric; the operator's communication mode applies). Arrays in the
 * operator's precision; u and lambda are consistent (assembled) vectors. */
int tn_epsdivdiv_vjp(tn_operator* op, const void* const* u_dev, const void* const* lambda_dev,
                     void* grad_logeta_cell_dev, void* const* grad_u_dev, void* stream);

/* Divergence B of velocity_level -> velocity_level-1 in Replace +
 * CommunicateAdditively mode (the same kernels and result as a
 * tn_divergence_create operator's tn_operator_apply) that allocates nothing:
 * its per-wedge scratch is a fixed 8 MiB static device array, enough for
 * velocity levels up to 5 (larger levels return TN_ERR_ARG). No counterpart in
 * the reference. For callers that cannot allocate device memory when they
 * apply the operator. Calls that overlap in time share the scratch and race;
 * the first call on a device does the set-up (looks up the scratch address)
 * and should come before any stream capture. The scratch used is the current
 * device's, so the shell's device must be current. u_dev: 3 velocity
 * components, p_dev: pressure. */
int tn_divergence_apply_noalloc(tn_shell* shell, int velocity_level, int precision, int bc_cmb, int bc_surface,
                                const void* const* u_dev, void* p_dev, void* stream);

/* Lumped k-weighted pressure mass diagonal, 6-point rule, interface-summed
 * (KMass with set_lumped_diagonal, src/terra/fe/wedge/operators/shell/
 * kmass.hpp:98-181; used with k = 1/eta as the Schur preconditioner,
 * apps/mantlecirculation/src/stokes_solver.hpp:559-584). */
int tn_kmass_lumped_diagonal(tn_shell* shell, int level, int precision, const void* k_dev, void* diag_dev,
                             void* stream);
/* dst = M src, vector mass matrix, interface-summed (VectorMass,
 * src/terra/fe/wedge/operators/shell/vector_mass.hpp:60-150). */
int tn_vector_mass_apply(tn_shell* shell, int level, int precision, const void* const* src_dev, void* const* dst_dev,
                         void* stream);

/* ---- multigrid transfers ----------------------------------------------------
 * fine += P coarse (ProlongationVecConstant in Add mode, src/terra/fe/wedge/
 * operators/shell/prolongation_constant.hpp:102-192) and coarse = R fine
 * including the coarse interface sum (RestrictionVecConstant,
 * restriction_constant.hpp:133-250). fine_level >= 1; ncomp 1..4. */
int tn_prolongate_add(tn_shell* shell, int fine_level, int precision, int ncomp, const void* const* coarse_dev,
                      void* const* fine_dev, void* stream);
int tn_restrict(tn_shell* shell, int fine_level, int precision, int ncomp, const void* const* fine_dev,
                void* const* coarse_dev, void* stream);
/* Linear transfers that interpolate affine functions exactly on the curved
 * shell (ProlongationLinear / RestrictionLinear, src/terra/fe/wedge/operators/
 * shell/prolongation_linear.hpp, restriction_linear.hpp, weights of
 * prolongation_linear_weights, src/terra/fe/wedge/shell/grid_transfer_linear.hpp:
 * 13-157), applied per component: fine += P coarse, and coarse = P^T (owned
 * fine) with the coarse interface sum. The weights of the fine level are
 * computed on first use (synchronous; before any stream capture). */
#define TN_TRANSFER_CONSTANT 0
#define TN_TRANSFER_LINEAR 1
int tn_prolongate_linear_add(tn_shell* shell, int fine_level, int precision, int ncomp, const void* const* coarse_dev,
                             void* const* fine_dev, void* stream);
int tn_restrict_linear(tn_shell* shell, int fine_level, int precision, int ncomp, const void* const* fine_dev,
                       void* const* coarse_dev, void* stream);

/* ---- nodal-vector kernels (VectorQ1Vec / VectorQ1Scalar, src/terra/linalg/
 * vector_q1.hpp:20-304; kernels/common/grid_operations.hpp) --------------- */
/* Sum every diamond-interface duplicate over its class (send_recv_with_plan,
 * src/terra/communication/shell/communication_plan.hpp:48-71). */
int tn_interface_sum(tn_shell* shell, int level, int precision, int ncomp, void* const* comps_dev, void* stream);
/* y = c0 + sum_i c[i] x_i, nterms in 0..3 (lincomb, vector.hpp). */
int tn_vec_lincomb(tn_shell* shell, int level, int precision, int ncomp, void* const* y_dev, double c0, int nterms,
                   const double* c, const void* const* x0_dev, const void* const* x1_dev, const void* const* x2_dev,
                   void* stream);
/* owned-node dot product accumulated in FP64 (masked_dot_product,
 * grid_operations.hpp:630-673). Synchronous on `stream`. */
int tn_vec_dot(tn_shell* shell, int level, int precision, int ncomp, const void* const* a_dev,
               const void* const* b_dev, double* result, void* stream);

/* A nodal vector of `level` (the VectorQ1Scalar / VectorQ1Vec constructors,
 * src/terra/linalg/vector_q1.hpp:20-120): ncomp arrays of the level's
 * (10, nl, nl, nr) nodes in `precision`, zero-filled, 256-byte aligned, their
 * device pointers written to comps_out. Synchronous. tn_vec_free releases
 * them (NULL entries are skipped). */
int  tn_vec_alloc(tn_shell* shell, int level, int precision, int ncomp, void** comps_out);
void tn_vec_free(int ncomp, void* const* comps);
/* Waits for everything queued on `stream` (the reference's Kokkos::fence()
 * after each apply); TN_ERR_CUDA if a launch or copy on it failed. */
int tn_sync(void* stream);

/* Uniform(-1, 1) values from SplitMix64 of (seed, canonical node, component):
 * the canonical node is the lowest lateral index of the node's duplicate class
 * times nr plus r, so interface duplicates receive equal values. Stands in for
 * randomize (grid_operations.hpp:748-773), whose stream depends on the backend. */
int tn_vec_random(tn_shell* shell, int level, int precision, int ncomp, uint64_t seed, void* const* comps_dev,
                  void* stream);

/* Remaining VectorLike operations (src/terra/linalg/vector.hpp:8-42; kernels in
 * src/terra/kernels/common/grid_operations.hpp). Entry-wise over all stored
 * nodes of ncomp (1..4) components of one level.
 *   invert_entries       y = 1 / y                     (grid_operations.hpp:232-253)
 *   scale_with_vector    y = y .* x                    (mult_elementwise_inplace, :255-273)
 *   max_abs_entry        max |a| over all entries      (:315-330); synchronous on `stream`
 *   has_nan_or_inf       1 if any entry is NaN or Inf  (:331-346); synchronous on `stream`
 *   swap                 a <-> b, entry-wise           (vector_q1.hpp swap_impl) */
int tn_vec_invert(tn_shell* shell, int level, int precision, int ncomp, void* const* y_dev, void* stream);
int tn_vec_scale(tn_shell* shell, int level, int precision, int ncomp, void* const* y_dev, const void* const* x_dev,
                 void* stream);
int tn_vec_max_abs(tn_shell* shell, int level, int precision, int ncomp, const void* const* a_dev, double* result,
                   void* stream);
int tn_vec_has_nan_or_inf(tn_shell* shell, int level, int precision, int ncomp, const void* const* a_dev, int* result,
                          void* stream);
int tn_vec_swap(tn_shell* shell, int level, int precision, int ncomp, void* const* a_dev, void* const* b_dev,
                void* stream);
/* Precision casts of n entries (the FP64 <-> FP32 boundary of the mixed-precision
 * solve; no counterpart in the FP64-only reference): direction TN_F64 means
 * FP64 in -> FP32 out, TN_F32 means FP32 in -> FP64 out. */
int tn_vec_cast(int64_t n, int direction, const void* in_dev, void* out_dev, void* stream);

/* ---- boundary treatment of right-hand sides --------------------------------
 * Node flags are the ShellBoundaryFlag values (src/terra/grid/shell/bit_masks.hpp:
 * 11-19): TN_FLAG_CMB on r = 0, TN_FLAG_SURFACE on r = nr-1, TN_FLAG_INNER else;
 * a node matches `flag` when it carries all of its bits (util/bit_masking.hpp:
 * 43-53; flag 0 matches no node of a shell). */
#define TN_FLAG_INNER 1
#define TN_FLAG_BOUNDARY 2
#define TN_FLAG_CMB 6
#define TN_FLAG_SURFACE 10
/* v = value on matching nodes, every component (assign_masked_else_keep_old,
 * src/terra/kernels/common/grid_operations.hpp:54-131; with value 0 the strong
 * Dirichlet step strong_algebraic_homogeneous_velocity_dirichlet_enforcement_
 * stokes_like, src/terra/fe/strong_algebraic_dirichlet_enforcement.hpp:114-123). */
int tn_vec_assign_masked(tn_shell* shell, int level, int precision, int ncomp, void* const* v_dev, int flag,
                         double value, void* stream);
/* On matching nodes of a 3-component vector: direction 0 rotates Cartesian
 * components into (normal, tangent 1, tangent 2), 1 rotates back
 * (cartesian_to_normal_tangential_in_place / normal_tangential_to_cartesian_in_place,
 * src/terra/linalg/trafo/local_basis_trafo_normal_tangential.hpp:34-186). */
int tn_vec_rotate_normal_tangential(tn_shell* shell, int level, int precision, void* const* v_dev, int flag,
                                    int direction, void* stream);
/* Remove the normal component on matching nodes (rotate, zero, rotate back:
 * strong_algebraic_freeslip_enforcement_in_place,
 * src/terra/fe/strong_algebraic_freeslip_enforcement.hpp:22-38). */
int tn_vec_freeslip_project(tn_shell* shell, int level, int precision, void* const* v_dev, int flag, void* stream);
/* The application's right-hand-side treatment (apps/mantlecirculation/src/
 * stokes_solver.hpp:662-671): the Dirichlet step on the boundary
 * get_shell_boundary_flag(bcs, DIRICHLET) returns, then the free-slip projection
 * on the one it returns for FREESLIP (src/terra/grid/shell/bit_masks.hpp:68-77:
 * the first match, CMB before SURFACE, so with Dirichlet on both boundaries only
 * the CMB rows are zeroed, as in the reference). u_dev: the 3 velocity
 * components of a right-hand side on `level`. */
int tn_stokes_rhs_enforce(tn_shell* shell, int level, int precision, int bc_cmb, int bc_surface, void* const* u_dev,
                          void* stream);

/* ---- stored element matrices and Galerkin coarse operators -----------------
 * set_stored_matrix_mode (epsilon_divdiv_kerngen.hpp:483-528) with
 * TN_STORED_FULL: assemble and keep the element matrices of the operator's
 * level from its FP64 coefficient (assemble_local_matrix, :2315-2392); the
 * apply then runs over the stored matrices with the boundary treatment of the
 * slow path (:1013-1242). TN_STORED_OFF returns to the matrix-free kernel.
 * Synchronous. */
int tn_operator_set_stored_matrix_mode(tn_operator* op, int mode, void* stream);
/* TwoGridGCA (src/terra/linalg/solvers/gca/gca.hpp:41-531): coarse (an
 * epsilon-div-div operator on level l-1 of the same shell) receives stored
 * matrices sum P^T A_f P over the 16 fine wedges of each coarse hex, A_f the
 * fine operator's stored matrices or its on-the-fly Neumann element matrices
 * (FP64 coefficient). The coarse operator applies in its own precision.
 * Synchronous. */
int tn_gca_build(tn_operator* fine, tn_operator* coarse, void* stream);
/* TwoGridGCA with its interpolation_mode argument (gca.hpp:72-78):
 * TN_TRANSFER_CONSTANT (InterpolationMode::Constant, tn_gca_build) or
 * TN_TRANSFER_LINEAR (InterpolationMode::Linear: P from the linear-transfer
 * weights, gca.hpp:231-243, :327-342). tensor_cores = 1 (the default of
 * tn_gca_build and of the solvers) is the fast build: over stored fine matrices
 * the batched 18 x 18 triple products P^T A P run on the FP64 tensor cores; over
 * on-the-fly fine matrices, which have the form k|J| (g g^T terms) of the wedge
 * gradients g, the product is formed directly from the gradients P^T g (the same
 * matrices to rounding). 0: the plain scalar triple product one fine wedge at a
 * time. Synchronous. */
int tn_gca_build_interpolated(tn_operator* fine, tn_operator* coarse, int interpolation, int tensor_cores,
                              void* stream);
/* GCAElementsCollector (src/terra/linalg/solvers/gca/gca_elements_collector.hpp:
 * 32-105): for each wedge of level `level`, the gradient of the nodal
 * coefficient k_dev in reference coordinates at the one-point rule's point; where
 * its norm exceeds 10 the ancestor cell level_range levels coarser is marked.
 * marks_dev: one byte per cell of level level - level_range (10, n-1, n-1,
 * nr-1), cleared first, 1 = marked. */
int tn_gca_mark_elements(tn_shell* shell, int level, int level_range, const double* k_dev, uint8_t* marks_dev,
                         void* stream);
/* set_stored_matrix_mode(Selective, level_range, GCAElements) (epsilon_divdiv_
 * kerngen.hpp:503-528; LocalMatrixStorage, local_matrix_storage.hpp:22-166):
 * the cells whose ancestor level_range levels coarser is marked in marks_dev
 * (as from tn_gca_mark_elements) take stored matrices, which a following
 * tn_gca_build fills; every other cell keeps the on-the-fly operator of the
 * operator's FP64 nodal coefficient (the slow path's per-cell choice, :1047-
 * 1060). A selective fine operator coarsens only into a selective coarse
 * operator with the same marks (TwoGridGCA builds the marked coarse cells, whose
 * fine children are all stored). Synchronous. */
int tn_operator_set_selective_matrices(tn_operator* op, int level_range, const uint8_t* marks_dev, void* stream);
/* cells with stored matrices (all cells in TN_STORED_FULL, the marked ones when
 * selective, 0 matrix-free) and the device bytes the stored matrices take (no
 * counterpart in the reference). */
int tn_operator_stored_cells(tn_operator* op, int64_t* stored_cells, int64_t* bytes);
/* get_local_matrix for every cell: host array (10, nl-1, nl-1, nr-1, 2, 18, 18),
 * dimension-wise ordering (row = node + 6 * component), without boundary
 * treatment. Synchronous. */
int tn_operator_copy_local_matrices(tn_operator* op, double* mats_host);

/* ---- solvers ----------------------------------------------------------------
 * Options of the Stokes FGMRES / velocity CG and of the multigrid
 * preconditioner (FGMRESOptions, fgmres.hpp:13-28; IterativeSolverParameters;
 * StokesSolverParameters, apps/mantlecirculation/src/parameters.hpp:154-184). */
typedef struct tn_solver_options {
    int      restart;                   /* FGMRES(m), 1..128 (30) */
    int      max_iterations;            /* outer iterations (300) */
    double   relative_tolerance;        /* 1e-8 */
    double   absolute_tolerance;        /* 1e-12 */
    int      chebyshev_order;           /* 2 */
    int      chebyshev_iterations;      /* pre- and post-smoothing steps (2) */
    int      power_iterations;          /* lambda_max estimate of D^-1 A (10) */
    int      num_vcycles;               /* V-cycles per preconditioner call (1) */
    int      coarse_max_iterations;     /* coarsest-level CG (50) */
    double   coarse_relative_tolerance; /* 1e-6 */
    double   coarse_absolute_tolerance; /* 1e-16 */
    int      gca;                       /* 1: Galerkin coarse operators on all coarse levels, 0: rediscretised,
                                           2: adaptive -- Galerkin matrices only on the cells below coarsest cells
                                           that GCAElementsCollector marks from the fine viscosity, rediscretised
                                           elsewhere (StokesSolverParameters::gca, parameters.hpp:166-176) (1) */
    int      mixed_precision;           /* 1: FP32 V-cycle inside the FP64 outer iteration (0) */
    uint64_t seed;                      /* power-iteration start vectors (12345) */
    int      normalize_pressure;        /* Stokes: subtract the owned-node pressure mean after the solve, as
                                           StokesContext::solve does (stokes_solver.hpp:684-690) (1) */
    int      project_pressure_mean;     /* Stokes: iterate on P K P, P removing the pressure mean, i.e. treat
                                           constant pressure as a null vector; not in the reference (0) */
    int      cuda_graphs;               /* Stokes: capture each Arnoldi step once and replay it as a CUDA
                                           graph (1) */
    int      smoother;                  /* multigrid smoother: TN_SMOOTHER_CHEBYSHEV (Chebyshev::solve_impl,
                                           chebyshev.hpp:102-176) or TN_SMOOTHER_JACOBI (damped Jacobi,
                                           Jacobi::solve_impl, jacobi.hpp:51-60, chebyshev_iterations steps)
                                           (TN_SMOOTHER_CHEBYSHEV) */
    double   jacobi_omega;              /* damped-Jacobi relaxation omega (1.0, the reference's default) */
    int      coarse_solver;             /* coarsest-level solve: TN_COARSE_PCG (the reference's PCG with
                                           coarse_max_iterations / coarse_relative_tolerance, pcg.hpp:81-169) or
                                           TN_COARSE_DENSE (the assembled coarsest operator inverted once at
                                           set-up, an exact solve by one dense product per V-cycle; coarsest
                                           levels up to 16384 unknowns) (TN_COARSE_PCG) */
    int      transfer;                  /* multigrid transfers and GCA interpolation: TN_TRANSFER_CONSTANT (the
                                           application's, stokes_solver.hpp:150-151) or TN_TRANSFER_LINEAR
                                           (tn_prolongate_linear_add / tn_restrict_linear, GCA with
                                           InterpolationMode::Linear) (TN_TRANSFER_CONSTANT) */
} tn_solver_options;
#define TN_SMOOTHER_CHEBYSHEV 0
#define TN_SMOOTHER_JACOBI 1
#define TN_COARSE_PCG 0
#define TN_COARSE_DENSE 1
void tn_solver_options_default(tn_solver_options* opts);
/* Stokes solve on velocity_level / velocity_level-1 (StokesContext,
 * apps/mantlecirculation/src/stokes_solver.hpp:325-609): FGMRES(m) with the
 * block-triangular preconditioner (block_preconditioner_2x2.hpp:205-221),
 * Schur block = inverse lumped KMass with k = 1/eta, velocity block = GMG
 * V-cycle (Chebyshev-Jacobi smoother, constant transfers, coarsest CG on
 * level 0). Exactly one of eta_nodal_dev (10,nl,nl,nr) and eta_cell_dev
 * (10,nl-1,nl-1,nr-1) is given (FP64, copied). k_schur_dev: nodal k on the
 * pressure level or NULL (then 1/eta at the pressure nodes; required with
 * eta_cell_dev). Levels 0..velocity_level of the shell form the hierarchy.
 * Synchronous setup (GCA build, diagonals, power iterations). */
int tn_stokes_solver_create(tn_shell* shell, int velocity_level, const double* eta_nodal_dev,
                            const double* eta_cell_dev, const double* k_schur_dev, int bc_cmb, int bc_surface,
                            const tn_solver_options* opts, void* stream, tn_solver** out);
/* Velocity-only CG (pcg.hpp:81-169) preconditioned by the same multigrid. */
int tn_velocity_solver_create(tn_shell* shell, int level, const double* eta_nodal_dev, const double* eta_cell_dev,
                              int bc_cmb, int bc_surface, const tn_solver_options* opts, void* stream,
                              tn_solver** out);
/* The velocity multigrid as a solver (Multigrid, src/terra/linalg/solvers/
 * multigrid.hpp:42-280, with the hierarchy the application builds, apps/
 * mantlecirculation/src/stokes_solver.hpp:351-557): levels 0..level of the
 * shell, smoother = Chebyshev(chebyshev_order, chebyshev_iterations,
 * power_iterations) or damped Jacobi (smoother, jacobi_omega), coarse =
 * coarse_solver, Galerkin or rediscretised coarse operators (gca). A solve runs
 * up to max_iterations times num_vcycles V-cycles from the initial guess in x,
 * recording the relative residual after each (the reference's statistics rows)
 * and stopping at relative_tolerance / absolute_tolerance. 3 components. */
int tn_multigrid_solver_create(tn_shell* shell, int level, const double* eta_nodal_dev, const double* eta_cell_dev,
                               int bc_cmb, int bc_surface, const tn_solver_options* opts, void* stream,
                               tn_solver** out);
void tn_solver_destroy(tn_solver* solver);
/* solve_impl(A, x, b): x_dev holds the initial guess and receives the
 * solution; 4 components (u_x, u_y, u_z, p) for a Stokes solver, 3 for a
 * velocity solver. Synchronous. TN_ERR_NOT_CONVERGED when the iteration limit
 * or a breakdown stopped it first (x_dev then holds the last iterate). */
int tn_solver_solve(tn_solver* solver, double* const* x_dev, const double* const* b_dev, void* stream);
/* Iterations (preconditioner applications), final relative residual
 * ||b - A x|| / ||b - A x0|| and whether the tolerance was met. */
int tn_solver_result(const tn_solver* solver, int* iterations, double* relative_residual, int* converged);
/* Stokes: final ||b - K x|| / ||b - K x0|| without the pressure-mean
 * projection (equal to the relative residual when the projection is off). */
int tn_solver_full_residual(const tn_solver* solver, double* relative_residual);
/* Relative residual per iteration (history[0] = 1); *length = entries available. */
int tn_solver_history(const tn_solver* solver, double* history_host, int capacity, int* length);
/* z = M^-1 v: the block preconditioner (Stokes, 4 components) or the
 * multigrid from z = 0 (velocity, 3 components). Synchronous. */
int tn_solver_precondition(tn_solver* solver, const double* const* v_dev, double* const* z_dev, void* stream);
/* num_vcycles V-cycles on A x = b of the velocity hierarchy in TN_F64 or TN_F32
 * (TN_F32 needs mixed_precision); x in/out. Synchronous. */
int tn_solver_vcycle(tn_solver* solver, int precision, void* const* x_dev, const void* const* b_dev, void* stream);
/* lambda_max(D^-1 A) of the Chebyshev smoother on level 1..fine. */
int tn_solver_level_lambda(tn_solver* solver, int level, double* lambda_max);
/* inverse diagonal used by the smoother on level 1..fine (3 components). */
int tn_solver_inverse_diagonal(tn_solver* solver, int level, double* const* out_dev, void* stream);
/* [iterations, initial residual, final residual] of the last coarsest CG. */
int tn_solver_coarse_stats(tn_solver* solver, double* stats3);
/* Adjoint gradient of J = 1/2 sum over owned velocity nodes |u - u_obs|^2
 * with respect to the per-cell log-viscosity of a Stokes solver created with
 * eta_cell_dev (no counterpart in the reference): x_dev is the forward
 * solution (4 components), u_obs_dev 3 components. One adjoint solve
 * K lambda = [u - u_obs; 0] (boundary rows enforced) with the solver's FGMRES,
 * then grad = -lambda_u^T dA/dlog(eta) u (tn_epsdivdiv_vjp). lambda_dev (4
 * components) receives the adjoint solution when not NULL. Synchronous;
 * TN_ERR_NOT_CONVERGED when the adjoint solve stopped early. */
int tn_stokes_misfit_gradient(tn_solver* solver, const double* const* x_dev, const double* const* u_obs_dev,
                              double* grad_logeta_cell_dev, double* const* lambda_dev, void* stream);
/* stored matrices of coarse level 0..fine-1 of the hierarchy, layout as
 * tn_operator_copy_local_matrices (adaptive GCA: the element matrices of the
 * rediscretised operator on unmarked cells). */
int tn_solver_level_matrices(tn_solver* solver, int level, double* mats_host);
/* stored cells and bytes of level 0..fine of the hierarchy (as
 * tn_operator_stored_cells). */
int tn_solver_level_storage(tn_solver* solver, int level, int64_t* stored_cells, int64_t* bytes);

/* ---- XDMF output that doubles as a checkpoint ------------------------------
 * The file format of the reference's XDMFOutput (src/terra/io/xdmf.hpp:13-148,
 * :293-512, :898-1060): per write, `<name>_<step>.bin` for every field and
 * `step_<step>.xmf`; the first write also writes geometry.bin (physical node
 * coordinates, 4- or 8-byte floats), topology.bin (two int64 wedges per hex
 * cell), checkpoint_metadata.bin and a README into `directory` (created if
 * missing). Binary order per diamond: r, y, x (fastest), component. A writer
 * covers one level of a shell; fields (1 or 3 components, device data in
 * `precision`, written with output_bytes = 4 or 8) are added before the first
 * write and read at every write. Synchronous. tn_xdmf_read restores a field of
 * step `step` into device memory (read_xdmf_checkpoint_grid). */
typedef struct tn_xdmf tn_xdmf;
int  tn_xdmf_create(tn_shell* shell, int level, const char* directory, int geometry_bytes, tn_xdmf** out);
int  tn_xdmf_add(tn_xdmf* x, const char* name, int precision, int ncomp, void* const* comps_dev, int output_bytes);
int  tn_xdmf_write(tn_xdmf* x, void* stream);
void tn_xdmf_destroy(tn_xdmf* x);
int  tn_xdmf_read(tn_shell* shell, int level, const char* directory, const char* name, int step, int precision,
                  int ncomp, void* const* comps_dev);

#ifdef __cplusplus
}
#endif
#endif /* TERRA_B200_H */
