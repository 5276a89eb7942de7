// Host-callable launchers of the sm_100a kernels. All pointers are device
// pointers; every launcher is asynchronous on `stream` and returns 0 or a
// negative launch error.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace tn {

// Kernel launches issued by the library (counter in runtime.cpp).
void     note_launch(int kernels = 1);
uint64_t launch_count();

// ----------------------------------------------------------------------------
// epsilon-div-div apply (epsdivdiv.cu)
// ----------------------------------------------------------------------------
template <typename T>
struct EddLaunch {
    int      nl = 0, nr = 0;
    const T* coords = nullptr;  // (10, nl, nl, 3)
    const T* radii  = nullptr;  // (nr)
    const T* k      = nullptr;  // nodal coefficient (10, nl, nl, nr) or nullptr
    const T* kq0    = nullptr;  // cell coefficient (10, nl-1, nl-1, nr-1) or nullptr
    const T* src[3] = {nullptr, nullptr, nullptr};
    T*       dst[3] = {nullptr, nullptr, nullptr};
    int      bc_cmb = 1, bc_surf = 1;  // 0 Neumann, 1 Dirichlet, 2 free-slip
    bool     diagonal = false;
    int      add      = 0;  // 0: dst = A src (owned nodes written), 1: dst += A src
    int      tile_y = 0, chunk_x = 0;  // 0: defaults
    int*     err = nullptr;            // device error word (bounded waits)
};
template <typename T>
int epsdivdiv_apply(const EddLaunch<T>& p, cudaStream_t stream);

// backward of the apply with respect to per-cell log-viscosity (adjoint.cu):
// grad[cell] (+)= lambda_e^T A_e(kq0[cell]) u_e
template <typename T>
struct VjpLaunch {
    int      nl = 0, nr = 0;
    const T* coords = nullptr;
    const T* radii  = nullptr;
    const T* kq0    = nullptr;
    const T* u[3]   = {nullptr, nullptr, nullptr};
    const T* lam[3] = {nullptr, nullptr, nullptr};
    T*       grad   = nullptr;  // (10, nl-1, nl-1, nr-1)
    int      bc_cmb = 1, bc_surf = 1;
    int      accumulate = 0;
};
template <typename T>
int epsdivdiv_vjp_logeta(const VjpLaunch<T>& p, cudaStream_t stream);

// ----------------------------------------------------------------------------
// Coupling blocks and mass matrices (stokes_coupling.cu). All accumulate into
// their outputs (callers zero them for Replace mode).
// ----------------------------------------------------------------------------
template <typename T>
struct CouplingLaunch {
    int      nl = 0, nr = 0;  // fine (velocity) level
    const T* coords = nullptr;
    const T* colgeo = nullptr;  // per-column wedge geometry (column_geometry_table)
    const T* radgeo = nullptr;  // per-radial-cell factors (radial_geometry_table)
    const T* radii  = nullptr;
    int      add    = 0;        // gradient: 1 accumulates into u_out, 0 overwrites
    T*       wedge_scratch = nullptr;  // 2 values per fine cell
    int      bc_cmb = 1, bc_surf = 1;
    const T* u[3]     = {nullptr, nullptr, nullptr};  // divergence input
    T*       p_out    = nullptr;                      // divergence output (coarse)
    const T* p_in     = nullptr;                      // gradient input (coarse)
    T*       u_out[3] = {nullptr, nullptr, nullptr};  // gradient output
};
// divergence accumulates into p_out (callers zero it for Replace); the
// gradient writes (or with add accumulates into) every node of u_out.
// Per radial cell rc of a level: alpha = 1/(2 r_mid), ib = 1/(6 hdr) and
// dfac = r_mid^2 hdr (r_mid, hdr: mid radius and half height of the cell),
// three values per cell.
template <typename T>
int radial_geometry_table(int nr, const T* radii, T* out, cudaStream_t stream);
template <typename T>
int divergence_apply(const CouplingLaunch<T>& p, cudaStream_t stream);
// e1, e2, e3 (columns of M^-T) and |det M| of both wedges of every lateral
// column, (10, nl-1, nl-1, 20)
template <typename T>
int column_geometry_table(int nl, const T* coords, T* out, cudaStream_t stream);
template <typename T>
int gradient_apply(const CouplingLaunch<T>& p, cudaStream_t stream);
template <typename T>
int kmass_lumped_add(int nl, int nr, const T* coords, const T* radii, const T* k, T* diag, cudaStream_t stream);
template <typename T>
int vector_mass_add(int nl, int nr, const T* coords, const T* radii, const T* const* src, T* const* dst,
                    cudaStream_t stream);

// ----------------------------------------------------------------------------
// Constant-weight grid transfers (transfer.cu). Levels given by the fine grid.
// prolongate_add: fine += P coarse (gather per fine node).
// restrict_owned: coarse = sum over owned fine neighbours (weights of
//                 prolongation_constant_weight); the interface sum follows.
// ----------------------------------------------------------------------------
template <typename T>
int prolongate_add(int nlf, int nrf, int ncomp, const T* const* coarse, T* const* fine, cudaStream_t stream);
template <typename T>
int restrict_owned(int nlf, int nrf, int ncomp, const uint8_t* owned_lat_fine, const T* const* fine, T* const* coarse,
                   cudaStream_t stream);

// Linear transfers (transfer_linear.cu): w holds two weights per fine node (linear_transfer_weights, FP64
// from the fine coordinates; FP32 copies for the FP32 V-cycle).
int linear_transfer_weights(int nlf, int nrf, const double* coords_fine, const double* radii_fine, double* w,
                            cudaStream_t stream);
template <typename T>
int prolongate_linear_add(int nlf, int nrf, int ncomp, const T* w, const T* const* coarse, T* const* fine,
                          cudaStream_t stream);
template <typename T>
int restrict_linear_owned(int nlf, int nrf, int ncomp, const uint8_t* owned_lat_fine, const T* w,
                          const T* const* fine, T* const* coarse, cudaStream_t stream);

// ----------------------------------------------------------------------------
// Interface sum over diamond-edge duplicates (vector_ops.cu).
// classes: offsets (num_classes + 1) into members (lateral indices).
// ----------------------------------------------------------------------------
struct IfaceTable {
    int            num_classes = 0;
    const int32_t* offset      = nullptr;
    const int32_t* members     = nullptr;
};
template <typename T>
int interface_sum(const IfaceTable& t, int nr, int ncomp, T* const* comps, cudaStream_t stream);

// ----------------------------------------------------------------------------
// BLAS-1 on nodal vectors of n elements per component (vector_ops.cu).
// ----------------------------------------------------------------------------
// y = c0 + sum_i c[i] * x_i  (0..3 terms), per component, ncomp components.
template <typename T>
int lincomb(int64_t n, int ncomp, T* const* y, T c0, int nterms, const T* c, const T* const* x0, const T* const* x1,
            const T* const* x2, cudaStream_t stream);
// y *= x elementwise
template <typename T>
int scale_inplace(int64_t n, int ncomp, T* const* y, const T* const* x, cudaStream_t stream);
// y = 1 / y
template <typename T>
int invert_inplace(int64_t n, int ncomp, T* const* y, cudaStream_t stream);
// out = sum over owned nodes and components of a * b, accumulated in double.
// owned_lat: (10, nl, nl) flags; the node's lateral index is i / nr.
template <typename T>
int masked_dot(int64_t n, int nr, int ncomp, const uint8_t* owned_lat, const T* const* a, const T* const* b,
               double* out_dev, double* partials, cudaStream_t stream);
// out = max |a| ; out_flags = 1 if any NaN/Inf
template <typename T>
int max_abs_and_nan(int64_t n, int ncomp, const T* const* a, double* out_dev, int* nan_dev, cudaStream_t stream);
// doubles of the shell's reduction scratch used by masked_dot / max_abs_and_nan partials
int reduction_partials_size();
// precision conversion
int convert_f64_to_f32(int64_t n, const double* in, float* out, cudaStream_t stream);
int convert_f32_to_f64(int64_t n, const float* in, double* out, cudaStream_t stream);

// ----------------------------------------------------------------------------
// Galerkin coarse operators and stored element matrices (gca.cu). Matrices
// are packed symmetric, 171 values per wedge, value-major: [w * 171 + p][cell].
// ----------------------------------------------------------------------------
int gca_values_per_cell();
// Selective storage (OperatorStoredMatrixMode::Selective, local_matrix_storage.hpp:22-166): matrices of the
// listed cells only, slot s of a [342][nslots] array holding cell cells[s]. For a build, cells / nslots
// name the coarse cells to build and fine_slot (fine cell -> slot, -1 none) / fine_stride the layout of the
// stored fine matrices; nullptr means every cell with slot = cell. A fine cell without a slot is reported
// to err (kDevBadLaunch).
struct GcaSlots {
    const int* cells       = nullptr;
    int        nslots      = 0;
    const int* fine_slot   = nullptr;
    int        fine_stride = 0;
    int*       err         = nullptr;
};
// coarse = sum P^T A_f P (fine level nlf, nrf); A_f from the nodal / cell
// coefficient (on-the-fly element matrices) or from stored fine matrices.
// linear_weights: the fine level's linear-transfer weights for InterpolationMode::Linear, or nullptr (Constant).
// tensor_cores: the fast build -- over on-the-fly fine matrices the rank form of the triple product, over
// stored ones the triple products as FP64 tensor-core tiles (mma m8n8k4); false: the plain scalar triple
// product one fine wedge at a time.
int gca_build(int nlf, int nrf, const double* coords_f, const double* radii_f, const double* k_f, const double* kq0_f,
              const double* fine_mats, double* coarse_mats, cudaStream_t st, const double* linear_weights = nullptr,
              bool tensor_cores = true, const GcaSlots& slots = GcaSlots{});
// element matrices of a level (the stored form of the on-the-fly operator), of every cell or of the listed
// ones; with base given, mats = base - element matrices
int element_matrices(int nl, int nr, const double* coords, const double* radii, const double* k, const double* kq0,
                     double* mats, cudaStream_t st, const int* cells = nullptr, int nslots = 0,
                     const double* base = nullptr);
// full[p][cells[s]] = compact[p][s]
int gca_scatter_slots(int nslots, const int* cells, const double* compact, int ncells, double* full, cudaStream_t st);
// GCAElementsCollector: marks[coarsest cell] = 1 for the coarsest ancestors (level_range halvings) of cells
// whose wedges have a reference-coordinate coefficient gradient above 10 (marks is not cleared)
int gca_mark_elements(int nl, int nr, const double* k, int level_range, uint8_t* marks, cudaStream_t st);
// bake Dirichlet masks / free-slip rotations of the boundary cells into mats
int gca_bake_boundary(int nl, int nr, const double* coords, const double* radii, int bc_cmb, int bc_surf, double* mats,
                      cudaStream_t st, const int* cells = nullptr, int nslots = 0);
// dst += A src with baked matrices
template <typename T>
int gca_apply_add(int nl, int nr, const T* mats, const T* const* src, T* const* dst, cudaStream_t st,
                  const int* cells = nullptr, int nslots = 0);
// dst += diag-mode(A) src with unbaked matrices
int gca_diag_add(int nl, int nr, const double* coords, const double* radii, int bc_cmb, int bc_surf,
                 const double* mats, const double* const* src, double* const* dst, cudaStream_t st,
                 const int* cells = nullptr, int nslots = 0);
int gca_to_f32(int64_t n, const double* in, float* out, cudaStream_t st);

// ----------------------------------------------------------------------------
// Solver kernels (solver_kernels.cu).
// A (block) vector is one allocation holding segments of components: a
// component of segment s starts at seg[s].offset + c * seg[s].stride and has
// seg[s].n valid entries; owned flags are per lateral node (entry / nr).
// ----------------------------------------------------------------------------
struct VecSeg {
    int64_t        offset = 0, n = 0, stride = 0;
    int            ncomp = 0, nr = 1;
    const uint8_t* owned = nullptr;
    uint64_t       rdiv  = 0;  // floor(2^40 / nr) + 1: lateral index of entry i = (i * rdiv) >> 40 (i < 2^25)
};
#ifdef __CUDACC__
#define TN_HOST_DEVICE __host__ __device__
#else
#define TN_HOST_DEVICE
#endif
TN_HOST_DEVICE inline uint64_t reciprocal_nr(int nr) { return (uint64_t(1) << 40) / static_cast<uint64_t>(nr) + 1; }

// Exact division by a fixed n through one multiply and shift:
// (i * (floor(2^40 / n) + 1)) >> 40 == i / n for 0 <= i < 2^40 / n, far above
// any level's entry count. Used to decode flat thread indices.
struct Decoder {
    int      n = 1;
    uint64_t m = 0;
    Decoder() = default;
    explicit Decoder(int n_) : n(n_), m(reciprocal_nr(n_)) {}
    TN_HOST_DEVICE int div(int i) const
    {
        return static_cast<int>((static_cast<uint64_t>(static_cast<uint32_t>(i)) * m) >> 40);
    }
};

// i = ((d * nlat + x) * nlat + y) * nrad + r  ->  (d, x, y, r) and the lateral
// column index (d * nlat + x) * nlat + y
TN_HOST_DEVICE inline void decode4(int i, const Decoder& rad, const Decoder& lat, int& d, int& x, int& y, int& r,
                                   int& col)
{
    col          = rad.div(i);
    r            = i - col * rad.n;
    const int dx = lat.div(col);
    y            = col - dx * lat.n;
    d            = lat.div(dx);
    x            = dx - d * lat.n;
}
struct VecDesc {
    int     nseg = 0;
    VecSeg  seg[2];
    int64_t total = 0;  // allocation length in elements (padding included)
};
// Per-block partials (solver_partials_size() doubles) and a zero-initialised
// completion counter that the last block resets.
struct RedScratch {
    double*   partials = nullptr;
    unsigned* counter  = nullptr;
};
constexpr int kMaxAxpy = 128;  // FGMRES restart limit (the list is a kernel parameter: 2 KB)
struct AxpyList {
    const double* z[kMaxAxpy];
    double        y[kMaxAxpy];
    int           m = 0;
};
struct CoarsePcgArgs {
    int            nl = 0, nr = 0;
    const double*  mats        = nullptr;  // baked stored matrices of the level
    const double*  mats_full   = nullptr;  // row-major copy (coarse_matrices_unpack), for the replicated kernel
    int            num_classes = 0;
    int            num_members = 0;  // off[num_classes]
    const int32_t* off = nullptr;
    const int32_t* mem = nullptr;
    const uint8_t* owned = nullptr;
    int64_t        n = 0, stride = 0;  // entries per component, component stride
    double*        x  = nullptr;       // in: initial guess, out: solution
    const double*  b  = nullptr;
    double*        r  = nullptr;
    double*        p  = nullptr;
    double*        ap = nullptr;
    double*        partials = nullptr;  // coarse_pcg_partials_size() doubles
    int            max_iter = 50;
    double         rtol = 1e-6, atol = 1e-16;
    double*        stats = nullptr;  // [iterations, initial residual, final residual] or nullptr
    // set by coarse_pcg: cells per CTA, bytes of the node table, matrices in shared memory
    int cells_per_cta = 0, node_bytes = 0, mats_in_smem = 0;
};
int solver_partials_size();
template <typename T>
int vec_dot(const VecDesc& L, const T* a, const T* b, double* out_dev, RedScratch rs, bool take_sqrt, cudaStream_t st);
// w -= (*h_sub) v_sub (when v_sub), then *out = <w, v_dot> or ||w|| (v_dot == nullptr)
int mgs_step(const VecDesc& L, double* w, const double* v_sub, const double* h_sub, const double* v_dot, double* out,
             RedScratch rs, cudaStream_t st);
// x += a p, r -= a ap with a = *s_an / *s_ad; *out = ||r|| (or -1 when
// |*s_ad| < DBL_MIN, in which case nothing is updated)
int cg_update(const VecDesc& L, double* x, double* r, const double* p, const double* ap, const double* s_an,
              const double* s_ad, double* out, RedScratch rs, cudaStream_t st);
// v -= scale * *s_dev on n entries
int sub_scalar(int64_t n, double* v, const double* s_dev, double scale, cudaStream_t st);
// p = z + (*s_num / *s_den) p (flat)
int p_update(int64_t n, double* p, const double* z, const double* s_num, const double* s_den, cudaStream_t st);
// y = x / *s_dev (flat over n entries)
template <typename T>
int scale_by_recip(int64_t n, T* y, const T* x, const double* s_dev, cudaStream_t st);
// Chebyshev step: d = alpha D^-1 (b - ax) [+ beta d], x += d (flat)
template <typename T>
int cheb_step(int64_t n, T* x, T* d, const T* b, const T* ax, const T* invdiag, T alpha, T beta, bool first,
              cudaStream_t st);
// y = c (a .* b) (flat)
template <typename T>
int vec_mul(int64_t n, T* y, const T* a, const T* b, T c, cudaStream_t st);
// x += sum_k y_k z_k (flat)
int multi_axpy(int64_t n, double* x, const AxpyList& list, cudaStream_t st);
// v = uniform(-1, 1) from SplitMix64 of (seed, canonical node id, component):
// duplicates of a node get the same value.
template <typename T>
int random_fill(int64_t n, int ncomp, T* const* comps, int nr, const int32_t* canon_lat, uint64_t seed,
                cudaStream_t st);
template <typename T>
int flag_nonfinite(int64_t n, const T* a, int* flag_dev, cudaStream_t st);
int widen_check(int64_t n, const float* in, double* out, int* flag_dev, cudaStream_t st);
int coarse_pcg(const CoarsePcgArgs& args, cudaStream_t st);
// decide and cache the launch configuration for a level (call outside graph capture)
int coarse_pcg_prepare(int nl, int nr, int num_classes, int num_members);
// 1 when the coarsest CG of this level runs the replicated kernel, which reads
// the row-major matrix copy made by coarse_matrices_unpack
int coarse_pcg_uses_full_matrices(int nl, int nr, int num_classes, int num_members);
// full[(w * 18 + a) * 18 + b][cell] = packed[w * 171 + pidx(a, b)][cell], nc cells
int coarse_matrices_unpack(int nc, const double* packed, double* full, cudaStream_t st);
int coarse_pcg_partials_size();

// Dense direct coarsest solve (coarse_dense.cu). Unknown (c, u) = c * nu + u; uid maps every stored node to
// its unique node, rep each unique node to its owned copy; vectors are 3 FP64 components `stride` apart.
constexpr int kDenseCoarseMaxUnknowns = 16384;  // 2 GB of FP64 inverse; the GEMV stages the rhs in shared memory
int dense_unit_vector(int64_t nodes, int64_t stride, int nu, const int32_t* uid, int dof, double* v, cudaStream_t st);
int dense_gather_column(int nu, int64_t stride, const int32_t* rep, const double* y, int col, double* K,
                        cudaStream_t st);
// in-place inverse of an SPD n x n matrix (Gauss-Jordan, no pivoting); colk: n doubles of scratch
int dense_invert_spd(int64_t n, double* A, double* colk, cudaStream_t st);
// kernel attributes for `unknowns` (call outside stream capture)
int dense_coarse_prepare(int unknowns);
// x = Kinv b (gathered at rep, scattered to every copy); y: 3 * nu doubles of scratch
int dense_coarse_solve(int64_t nodes, int64_t stride, int nu, const int32_t* uid, const int32_t* rep,
                       const double* Kinv, const double* b, double* y, double* x, cudaStream_t st);

}  // namespace tn
