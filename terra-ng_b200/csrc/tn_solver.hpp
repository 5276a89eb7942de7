// Solver layer behind the C ABI: the velocity multigrid hierarchy (GCA or
// rediscretised coarse operators, Chebyshev-Jacobi smoothing, constant
// transfers, coarsest-grid CG), the block-triangular Stokes preconditioner and
// FGMRES, in FP64 or with an FP32 V-cycle inside the FP64 outer iteration.
#pragma once

#include <vector>

#include "tn_runtime.hpp"

namespace tn {

VecDesc velocity_desc(const DeviceLevel& L);
VecDesc scalar_desc(const DeviceLevel& L);
VecDesc stokes_desc(const DeviceLevel& Lu, const DeviceLevel& Lp);

// A zero-initialised vector allocation with its segment layout.
template <typename T>
struct DVec {
    DevBuf  buf;
    VecDesc d;
    void    alloc(const VecDesc& desc);
    T*      data() const { return buf.as<T>(); }
    T*      comp(int s, int c) const { return data() + d.seg[s].offset + c * d.seg[s].stride; }
    int     ncomp() const;
    void    comps(T** out) const;  // all components, segment by segment
    int64_t total() const { return d.total; }
};

// Reduction scratch, device scalars, a device flag and a pinned host mirror.
struct Scratch {
    DevBuf  partials, counter, scal, flag;
    double* host     = nullptr;  // kScalars doubles + flag, pinned
    static constexpr int kScalars = 256;
    Scratch();
    ~Scratch();
    Scratch(const Scratch&)            = delete;
    Scratch& operator=(const Scratch&) = delete;
    RedScratch rs() const { return {partials.as<double>(), counter.as<unsigned>()}; }
    double*    s(int i) const { return scal.as<double>() + i; }
    int*       flag_dev() const { return flag.as<int>(); }
    // copy scal[0, n) and the flag to the host and wait
    void fetch(int n, cudaStream_t st);
    int  host_flag() const { return *reinterpret_cast<const int*>(host + kScalars); }
};

struct MgOptions {
    int      cheb_order = 2, cheb_iters = 2, power_iters = 10, num_vcycles = 1;
    int      coarse_max_iter = 50;
    double   coarse_rtol = 1e-6, coarse_atol = 1e-16;
    int      gca  = 1;      // 1: Galerkin coarse operators on every coarse level; 0: rediscretised
    bool     fp32 = false;  // FP32 V-cycle (coarsest solve stays FP64)
    uint64_t seed = 12345;  // power-iteration start vectors
    int      smoother     = 0;    // 0: Chebyshev (cheb_order, cheb_iters), 1: damped Jacobi (cheb_iters steps)
    double   jacobi_omega = 1.0;  // Jacobi relaxation
    int      coarse_dense = 0;    // 0: coarsest CG (the reference's PCG); 1: dense inverse built once, exact solve
    int      transfer     = 0;    // 0: constant transfers (the application's), 1: linear (also in the GCA build)
};

// Velocity multigrid (Multigrid, multigrid.hpp:216-432) over levels 0..fine of
// a shell, built from an FP64 fine operator.
class VelocityMultigrid {
  public:
    VelocityMultigrid(const Shell* sh, const EpsDivDivOp& fine, const MgOptions& o, Scratch& scratch,
                      cudaStream_t st);
    // num_vcycles V-cycles on A x = b; x, b are velocity vectors (velocity_desc
    // layout) of the fine level in the precision of the call.
    // x_zero: x holds zeros on entry (the first smoothing step then skips A x)
    void solve64(double* x, const double* b, cudaStream_t st, bool x_zero = false);
    void solve32(float* x, const float* b, cudaStream_t st, bool x_zero = false);
    double           lambda(int l) const { return lambda_.at(l); }
    const DVec<double>& inv_diag(int l) const { return w64_.invdiag.at(l); }
    EpsDivDivOp&     op64(int l) { return *ops64_.at(l); }
    int              fine_level() const { return fine_; }
    const MgOptions& options() const { return opt_; }
    // statistics of the last coarsest solve [iterations, initial, final residual] (synchronises)
    void coarse_stats(double* out3, cudaStream_t st);
    // power iteration on D^-1 A of level l from the seeded start vector (power_iteration.hpp:15-57)
    double power_iteration(int l, int iterations, uint64_t seed, cudaStream_t st);
    // solve64 / solve32 on the caller's component arrays (3 x nodes of the fine level)
    template <typename T>
    void solve_external(T* const* x, const T* const* b, cudaStream_t st);

  private:
    template <typename T>
    struct Work {
        std::vector<DVec<T>> r, e, tmp, d, invdiag;
    };
    template <typename T>
    Work<T>& work();
    template <typename T>
    void apply(int l, const T* x, T* y, cudaStream_t st);
    template <typename T>
    void smooth(int l, T* x, const T* b, cudaStream_t st, bool x_zero);
    template <typename T>
    void vcycle(int l, T* x, const T* b, cudaStream_t st, bool x_zero);
    template <typename T>
    void coarse_solve(T* x, const T* b, cudaStream_t st);
    void build_dense_coarse(cudaStream_t st);  // kinv_ = inverse of the assembled coarsest operator

    const Shell*                              sh_;
    int                                       fine_;
    MgOptions                                 opt_;
    Scratch&                                  scratch_;
    std::vector<std::unique_ptr<EpsDivDivOp>> ops64_;     // levels 0..fine
    std::vector<std::unique_ptr<EpsDivDivOp>> ops32_;     // on-the-fly FP32 operators (null where stored)
    std::vector<double>                       lambda_;
    Work<double>                              w64_;
    Work<float>                               w32_;
    DVec<double>                              cx_, cb_, cr_, cp_, cap_;  // coarsest CG vectors
    DevBuf                                    cpart_, cstats_;
    DevBuf                                    cfull_;  // row-major coarsest matrices (replicated CG)
    DevBuf                                    kinv_, kuid_, krep_, ky_;  // dense coarsest solve
    int                                       knu_ = 0;                  // unique coarsest nodes
    DVec<double>                              ext64_[2];
    DVec<float>                               ext32_[2];
};

struct StokesOptions {
    int       restart = 30, max_iter = 300;
    double    rtol = 1e-8, atol = 1e-12;
    bool      normalize_pressure = true;
    bool      project_pressure_mean = false;  // treat constant pressure as a null vector (see solve())
    bool      use_graphs = true;              // replay each Arnoldi step as a captured CUDA graph
    MgOptions mg;
};

// FGMRES (fgmres.hpp:109-373) on the Stokes block operator with the
// block-triangular preconditioner (block_preconditioner_2x2.hpp:205-221):
// Schur block = inverse lumped k-mass with k = 1/eta (stokes_solver.hpp:559-584),
// velocity block = the multigrid V-cycle.
class StokesSolver {
  public:
    // eta: viscosity on the velocity level, nodal or per cell (FP64 device).
    // k_schur: nodal 1/eta on the pressure level or nullptr (nodal eta only:
    // taken from eta at the pressure nodes).
    StokesSolver(const Shell* sh, int vlevel, const double* eta_nodal, const double* eta_cell, const double* k_schur,
                 int bc_cmb, int bc_surf, const StokesOptions& o, cudaStream_t st);
    ~StokesSolver();
    StokesSolver(const StokesSolver&)            = delete;
    StokesSolver& operator=(const StokesSolver&) = delete;
    // u, p in/out (initial guess, solution); f_u, f_p right-hand side; caller's
    // component arrays. Synchronous. Returns true when the tolerance was met.
    bool solve(double* const* u, double* p, const double* const* fu, const double* fp, cudaStream_t st);
    // z = M^-1 v for 4-component vectors in the caller's layout
    void precondition_external(const double* const* v, double* const* z, cudaStream_t st);
    // dJ/d log(eta_cell) of J = 1/2 sum over owned nodes |u - u_obs|^2 at the
    // forward solution x (4 components): one adjoint solve K lambda = [u -
    // u_obs; 0] (K is symmetric) and the backward kernel, grad = -lambda_u^T
    // dA/dlog(eta) u. Needs a per-cell viscosity. lambda (4 components) is
    // returned when not null. Returns whether the adjoint solve converged.
    bool misfit_gradient(const double* const* x, const double* const* u_obs, double* grad_cell,
                         double* const* lambda, cudaStream_t st);

    std::vector<double> history;  // relative residual estimates, history[0] = 1
    int                 iterations = 0;
    double              final_relres = 0.0;
    double              full_relres  = 0.0;  // ||b - K x|| / ||b - K x0|| without the pressure-mean projection
    bool                converged = false;
    VelocityMultigrid&  mg() { return *mg_; }
    const StokesOptions& options() const { return opt_; }

  private:
    static constexpr int kH0   = 2;                      // Hessenberg column in scalar slots kH0..
    static constexpr int kProj = Scratch::kScalars - 1;  // scalar slot of the pressure-mean projection
    bool solve_internal(cudaStream_t st);  // x_ (initial guess -> solution), b_
    void step_body(int j, cudaStream_t st);
    void arnoldi_tail(int j, cudaStream_t st);
    void run_step(int j, cudaStream_t st);
    void precondition(const DVec<double>& v, DVec<double>& z, cudaStream_t st);
    void stokes_apply(const DVec<double>& x, DVec<double>& y, cudaStream_t st);
    void copy_in(DVec<double>& v, const double* const* u, const double* p, cudaStream_t st);
    void copy_out(const DVec<double>& v, double* const* u, double* p, cudaStream_t st);
    void remove_pressure_mean(DVec<double>& v, int slot, cudaStream_t st);

    const Shell*                       sh_;
    int                                vlevel_;
    StokesOptions                      opt_;
    Scratch                            scratch_;
    StokesOp                           K_;
    GradientOp                         BT_;
    DVec<double>                       inv_schur_;  // pressure level
    DVec<double>                       ones_p_;     // pressure level, for the mean
    int64_t                            num_owned_p_ = 0;
    std::unique_ptr<VelocityMultigrid> mg_;
    VecDesc                            blk_;
    DVec<double>                       x_, b_, r_, w_, t_;
    std::vector<DVec<double>>          V_, Z_;
    DVec<float>                        t32_, z32_;
    std::vector<cudaGraphExec_t>       graphs_;
    std::vector<int>                   graph_kernels_;  // kernels captured in each graph
    cudaStream_t                       ws_ = nullptr;
};

struct VelocitySolverOptions {
    int       max_iter = 100;
    double    rtol = 1e-8, atol = 1e-16;
    bool      multigrid_only = false;  // Multigrid::solve_impl: repeated V-cycles (num_vcycles each) instead of CG
    MgOptions mg;
};

// PCG (pcg.hpp:81-169) on the epsilon-div-div operator with the velocity
// multigrid as preconditioner, each application starting from z = 0; or, with
// multigrid_only, the multigrid as the solver (Multigrid::solve_impl,
// multigrid.hpp:216-280): V-cycles from the caller's initial guess with the
// residual recorded after each, stopping at the relative tolerance.
class VelocitySolver {
  public:
    VelocitySolver(const Shell* sh, int level, const double* eta_nodal, const double* eta_cell, int bc_cmb,
                   int bc_surf, const VelocitySolverOptions& o, cudaStream_t st);
    bool solve(double* const* u, const double* const* f, cudaStream_t st);
    // z = MG(0; v) on the caller's arrays
    void precondition_external(const double* const* v, double* const* z, cudaStream_t st);

    std::vector<double> history;
    int                 iterations = 0;
    double              final_relres = 0.0;
    bool                converged = false;
    VelocityMultigrid&  mg() { return *mg_; }

  private:
    void precondition(cudaStream_t st);  // z_ = MG(z_; r_)

    const Shell*                       sh_;
    VelocitySolverOptions              opt_;
    Scratch                            scratch_;
    EpsDivDivOp                        A_;
    std::unique_ptr<VelocityMultigrid> mg_;
    VecDesc                            vd_;
    DVec<double>                       x_, b_, r_, z_, p_, ap_;
    DVec<float>                        r32_, z32_;
};

int enforce_velocity_bcs(int nl, int nr, const double* coords, int bc_cmb, int bc_surf, double* const* v,
                         cudaStream_t st);

// coefficient of a coarser level: nodal injection (optionally reciprocal) or
// the mean of the 8 child cells (solver_kernels.cu)
int coefficient_inject(int nlc, int nrc, const double* fine, double* coarse, bool reciprocal, cudaStream_t st);
int cell_coefficient_average(int nlc, int nrc, const double* fine, double* coarse, cudaStream_t st);

}  // namespace tn
