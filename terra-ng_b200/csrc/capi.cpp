// extern "C" boundary (include/terra_b200.h). Exceptions never cross it: every
// entry point converts them into a status code plus a thread-local message.
#include <cstring>
#include <string>

#include "../../include/terra_b200.h"
#include "tn_boundary.hpp"
#include "tn_solver.hpp"

struct tn_shell {
    std::unique_ptr<tn::Shell> impl;
};
struct tn_operator {
    std::unique_ptr<tn::Operator> op;
};
struct tn_xdmf {
    tn::Xdmf* impl = nullptr;
    ~tn_xdmf() { tn::xdmf_destroy(impl); }
};
struct tn_solver {
    tn_shell*                           shell = nullptr;
    std::unique_ptr<tn::StokesSolver>   stokes;
    std::unique_ptr<tn::VelocitySolver> velocity;
    tn::VelocityMultigrid&              mg() { return stokes ? stokes->mg() : velocity->mg(); }
};

namespace {
thread_local std::string g_last_error;

template <typename F>
int guarded(F&& f)
{
    try {
        g_last_error.clear();
        f();
        return TN_OK;
    } catch (const tn::Error& e) {
        g_last_error = e.what();
        return e.code;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return TN_ERR_ARG;
    } catch (...) {
        g_last_error = "unknown error";
        return TN_ERR_ARG;
    }
}

void need(bool cond, const char* msg)
{
    if (!cond) throw tn::Error(tn::kErrArg, msg);
}

int precision_size(int p)
{
    if (p == TN_F64) return 8;
    if (p == TN_F32) return 4;
    throw tn::Error(tn::kErrArg, "precision must be TN_F64 or TN_F32");
}

cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }
}  // namespace

namespace {
void check_bcs(int bc_cmb, int bc_surface)
{
    need(bc_cmb >= 0 && bc_cmb <= 2 && bc_surface >= 0 && bc_surface <= 2, "invalid boundary condition");
}

void init_edd(tn::EpsDivDivOp& e, tn::Shell* sh, int level, int precision, const void* k_nodal_dev,
              const void* k_cell_dev, int bc_cmb, int bc_surface, int diagonal)
{
    need((k_nodal_dev == nullptr) != (k_cell_dev == nullptr), "exactly one of k_nodal / k_cell must be given");
    check_bcs(bc_cmb, bc_surface);
    const int   es = precision_size(precision);
    const auto& L  = sh->level(level);
    need(L.nr() >= 3, "the operator needs at least two radial layers");
    e.shell     = sh;
    e.level     = level;
    e.precision = precision;
    e.q0        = k_cell_dev != nullptr;
    e.bc_cmb    = bc_cmb;
    e.bc_surf   = bc_surface;
    e.diagonal  = diagonal != 0;
    const size_t n = static_cast<size_t>(e.q0 ? L.cells() : L.nodes());
    e.k.alloc(n * es);
    tn::cuda_check(cudaMemcpy(e.k.get(), e.q0 ? k_cell_dev : k_nodal_dev, n * es, cudaMemcpyDeviceToDevice),
                   "copy coefficient");
}

template <typename Op>
void init_coupling(Op& o, tn::Shell* sh, int level, int precision, int bc_cmb, int bc_surface)
{
    check_bcs(bc_cmb, bc_surface);
    precision_size(precision);
    sh->level(level);
    need(level >= 1, "the velocity level needs a coarser pressure level below it");
    o.shell     = sh;
    o.level     = level;
    o.precision = precision;
    o.bc_cmb    = bc_cmb;
    o.bc_surf   = bc_surface;
}

tn::MgOptions mg_options(const tn_solver_options& o)
{
    tn::MgOptions m;
    m.cheb_order      = o.chebyshev_order;
    m.cheb_iters      = o.chebyshev_iterations;
    m.power_iters     = o.power_iterations;
    m.num_vcycles     = o.num_vcycles;
    m.coarse_max_iter = o.coarse_max_iterations;
    m.coarse_rtol     = o.coarse_relative_tolerance;
    m.coarse_atol     = o.coarse_absolute_tolerance;
    m.gca             = o.gca;
    m.fp32            = o.mixed_precision != 0;
    m.seed            = o.seed;
    m.smoother        = o.smoother;
    m.jacobi_omega    = o.jacobi_omega;
    m.coarse_dense    = o.coarse_solver == TN_COARSE_DENSE ? 1 : 0;
    m.transfer        = o.transfer == TN_TRANSFER_LINEAR ? 1 : 0;
    need(o.transfer == TN_TRANSFER_CONSTANT || o.transfer == TN_TRANSFER_LINEAR, "unknown transfer");
    need(o.coarse_solver == TN_COARSE_PCG || o.coarse_solver == TN_COARSE_DENSE, "unknown coarse solver");
    need(o.gca == 0 || o.gca == 1 || o.gca == 2, "gca must be 0, 1 or 2");
    need(o.smoother == TN_SMOOTHER_CHEBYSHEV || o.smoother == TN_SMOOTHER_JACOBI, "unknown smoother");
    need(o.jacobi_omega > 0.0, "jacobi_omega must be positive");
    return m;
}

// stored packed matrices -> (cells, 2, 18, 18) full symmetric host array
void unpack_matrices(const tn::EpsDivDivOp& op, double* mats_host)
{
    need((op.stored && op.mats.get()) || (op.selective && op.sel_built), "the operator has no stored matrices");
    const int64_t       nc = op.lvl().cells();
    std::vector<double> packed(static_cast<size_t>(tn::gca_values_per_cell()) * nc);
    tn::DevBuf          eff;  // selective storage: stored matrices on marked cells, element matrices elsewhere
    if (op.selective) {
        op.effective_matrices(eff, nullptr);
        tn::cuda_check(cudaStreamSynchronize(nullptr), "assemble matrices");
    }
    tn::cuda_check(cudaMemcpy(packed.data(), op.selective ? eff.get() : op.mats.get(), packed.size() * sizeof(double),
                              cudaMemcpyDeviceToHost),
                   "copy matrices");
    for (int64_t c = 0; c < nc; ++c)
        for (int w = 0; w < 2; ++w) {
            int p = 0;
            for (int i = 0; i < 18; ++i)
                for (int j = i; j < 18; ++j, ++p) {
                    const double v                             = packed[static_cast<size_t>(w * 171 + p) * nc + c];
                    mats_host[((c * 2 + w) * 18 + i) * 18 + j] = v;
                    mats_host[((c * 2 + w) * 18 + j) * 18 + i] = v;
                }
        }
}

tn::EpsDivDivOp* as_edd(tn_operator* op)
{
    auto* e = dynamic_cast<tn::EpsDivDivOp*>(op->op.get());
    if (!e) throw tn::Error(tn::kErrArg, "not an epsilon-div-div operator");
    return e;
}
}  // namespace

namespace {
template <typename F>
int dispatch_prec(int precision, F&& f)
{
    precision_size(precision);
    return precision == TN_F64 ? f(double{}) : f(float{});
}
void check_comps(int ncomp, const void* p)
{
    need(p != nullptr, "NULL argument");
    need(ncomp >= 1 && ncomp <= 4, "ncomp must be 1..4");
}
}  // namespace

namespace {
void max_abs_nan(tn_shell* shell, int level, int precision, int ncomp, const void* const* a_dev, double* mx, int* nan,
                 void* stream)
{
    check_comps(ncomp, a_dev);
    const auto& L   = shell->impl->level(level);
    double*     red = shell->impl->red.as<double>();
    int*        flag = reinterpret_cast<int*>(red + tn::reduction_partials_size() + 4);
    tn::cuda_check(cudaMemsetAsync(flag, 0, sizeof(int), as_stream(stream)), "clear flag");
    const int rc = dispatch_prec(precision, [&](auto t) {
        using T = decltype(t);
        return tn::max_abs_and_nan<T>(L.nodes(), ncomp, reinterpret_cast<const T* const*>(a_dev), red, flag,
                                      as_stream(stream));
    });
    if (rc) throw tn::Error(tn::kErrCuda, "max-abs launch failed");
    double h_mx = 0.0;
    int    h_nan = 0;
    tn::cuda_check(cudaMemcpyAsync(&h_mx, red, sizeof(double), cudaMemcpyDeviceToHost, as_stream(stream)), "readback");
    tn::cuda_check(cudaMemcpyAsync(&h_nan, flag, sizeof(int), cudaMemcpyDeviceToHost, as_stream(stream)), "readback");
    tn::cuda_check(cudaStreamSynchronize(as_stream(stream)), "max-abs sync");
    if (mx) *mx = h_mx;
    if (nan) *nan = h_nan != 0;
}
}  // namespace

namespace {
void rotate(tn_shell* shell, int level, int precision, void* const* v_dev, int flag, int mode, void* stream)
{
    need(shell, "NULL shell");
    check_comps(3, v_dev);
    need(flag >= 0 && flag < 256, "flag must be a ShellBoundaryFlag value");
    const auto& L  = shell->impl->level(level);
    const int   rc = dispatch_prec(precision, [&](auto t) {
        using T = decltype(t);
        return tn::rotate_normal_tangential<T>(L.nodes(), L.nr(), L.coords<T>(), reinterpret_cast<T* const*>(v_dev),
                                               flag, mode, as_stream(stream));
    });
    if (rc) throw tn::Error(tn::kErrCuda, "rotation launch failed");
}
int shell_boundary_flag(int bc_cmb, int bc_surface, int bcf)
{
    if (bc_cmb == bcf) return tn::kFlagCMB;
    if (bc_surface == bcf) return tn::kFlagSurface;
    return 0;
}
}  // namespace


extern "C" {

const char* tn_last_error(void) { return g_last_error.c_str(); }
const char* tn_version(void) { return "terra_b200 0.1 (sm_100a)"; }

uint64_t tn_kernel_launch_count(void) { return tn::launch_count(); }

int tn_shell_create(int lat_level, int rad_level, int num_levels, double r_min, double r_max, tn_shell** out)
{
    return guarded([&] {
        need(out != nullptr, "out is NULL");
        auto s  = new tn_shell;
        try {
            s->impl = tn::make_shell(lat_level, rad_level, num_levels, r_min, r_max);
        } catch (...) {
            delete s;
            throw;
        }
        *out = s;
    });
}

void tn_shell_destroy(tn_shell* shell) { delete shell; }

int tn_shell_num_levels(const tn_shell* shell, int* num_levels)
{
    return guarded([&] {
        need(shell && num_levels, "NULL argument");
        *num_levels = static_cast<int>(shell->impl->levels.size());
    });
}

int tn_shell_level_dims(const tn_shell* shell, int level, int* nl, int* nr)
{
    return guarded([&] {
        need(shell && nl && nr, "NULL argument");
        const auto& L = shell->impl->level(level);
        *nl           = L.nl();
        *nr           = L.nr();
    });
}

int tn_shell_copy_coords(const tn_shell* shell, int level, double* coords_host)
{
    return guarded([&] {
        need(shell && coords_host, "NULL argument");
        const auto& h = shell->impl->level(level).host;
        std::memcpy(coords_host, h.coords.data(), h.coords.size() * sizeof(double));
    });
}

int tn_shell_copy_radii(const tn_shell* shell, int level, double* radii_host)
{
    return guarded([&] {
        need(shell && radii_host, "NULL argument");
        const auto& h = shell->impl->level(level).host;
        std::memcpy(radii_host, h.radii.data(), h.radii.size() * sizeof(double));
    });
}

int tn_shell_copy_ownership(const tn_shell* shell, int level, uint8_t* owned_host)
{
    return guarded([&] {
        need(shell && owned_host, "NULL argument");
        const auto& h = shell->impl->level(level).host;
        for (size_t i = 0; i < h.owned_lat.size(); ++i)
            std::memset(owned_host + i * h.nr, h.owned_lat[i], static_cast<size_t>(h.nr));
    });
}

int tn_shell_copy_boundary_mask(const tn_shell* shell, int level, uint8_t* mask_host)
{
    return guarded([&] {
        need(shell && mask_host, "NULL argument");
        const auto& h = shell->impl->level(level).host;
        for (size_t i = 0; i < h.owned_lat.size(); ++i)
            for (int r = 0; r < h.nr; ++r) mask_host[i * h.nr + r] = tn::boundary_flag(r, h.nr);
    });
}

int tn_shell_duplicate_classes(const tn_shell* shell, int level, int32_t* class_of_lat_host, int* num_classes)
{
    return guarded([&] {
        need(shell && class_of_lat_host && num_classes, "NULL argument");
        const auto& h = shell->impl->level(level).host;
        for (size_t i = 0; i < h.owned_lat.size(); ++i) class_of_lat_host[i] = -1;
        const int nc = static_cast<int>(h.dup_offset.size()) - 1;
        for (int c = 0; c < nc; ++c)
            for (int m = h.dup_offset[c]; m < h.dup_offset[c + 1]; ++m) class_of_lat_host[h.dup_members[m]] = c;
        *num_classes = nc;
    });
}

int tn_mesh_generate_host(int lat_level, int rad_level, double r_min, double r_max, double* coords_host,
                          double* radii_host, uint8_t* owned_lat_host, int32_t* class_of_lat_host, int* num_classes)
{
    return guarded([&] {
        tn::ShellLevel h;
        try {
            h = tn::make_shell_level(lat_level, rad_level, r_min, r_max);
        } catch (const std::invalid_argument& e) {
            throw tn::Error(tn::kErrArg, e.what());
        }
        if (coords_host) std::memcpy(coords_host, h.coords.data(), h.coords.size() * sizeof(double));
        if (radii_host) std::memcpy(radii_host, h.radii.data(), h.radii.size() * sizeof(double));
        if (owned_lat_host) std::memcpy(owned_lat_host, h.owned_lat.data(), h.owned_lat.size());
        const int nc = static_cast<int>(h.dup_offset.size()) - 1;
        if (class_of_lat_host) {
            for (size_t i = 0; i < h.owned_lat.size(); ++i) class_of_lat_host[i] = -1;
            for (int c = 0; c < nc; ++c)
                for (int m = h.dup_offset[c]; m < h.dup_offset[c + 1]; ++m) class_of_lat_host[h.dup_members[m]] = c;
        }
        if (num_classes) *num_classes = nc;
    });
}

int tn_shell_check_device_error(tn_shell* shell, int* code)
{
    return guarded([&] {
        need(shell && code, "NULL argument");
        tn::cuda_check(cudaDeviceSynchronize(), "synchronize");
        int v = 0;
        tn::cuda_check(cudaMemcpy(&v, shell->impl->err.get(), sizeof(int), cudaMemcpyDeviceToHost), "read error");
        tn::cuda_check(cudaMemset(shell->impl->err.get(), 0, sizeof(int)), "clear error");
        *code = v;
    });
}


int tn_epsdivdiv_create(tn_shell* shell, int level, int precision, const void* k_nodal_dev, const void* k_cell_dev,
                        int bc_cmb, int bc_surface, int diagonal, tn_operator** out)
{
    return guarded([&] {
        need(shell && out, "NULL argument");
        auto e = std::make_unique<tn::EpsDivDivOp>();
        init_edd(*e, shell->impl.get(), level, precision, k_nodal_dev, k_cell_dev, bc_cmb, bc_surface, diagonal);
        e->prepare_penalty(nullptr);
        auto o = new tn_operator;
        o->op  = std::move(e);
        *out   = o;
    });
}

int tn_divergence_create(tn_shell* shell, int velocity_level, int precision, int bc_cmb, int bc_surface,
                         tn_operator** out)
{
    return guarded([&] {
        need(shell && out, "NULL argument");
        auto b = std::make_unique<tn::DivergenceOp>();
        init_coupling(*b, shell->impl.get(), velocity_level, precision, bc_cmb, bc_surface);
        auto o = new tn_operator;
        o->op  = std::move(b);
        *out   = o;
    });
}

int tn_gradient_create(tn_shell* shell, int velocity_level, int precision, int bc_cmb, int bc_surface,
                       tn_operator** out)
{
    return guarded([&] {
        need(shell && out, "NULL argument");
        auto b = std::make_unique<tn::GradientOp>();
        init_coupling(*b, shell->impl.get(), velocity_level, precision, bc_cmb, bc_surface);
        auto o = new tn_operator;
        o->op  = std::move(b);
        *out   = o;
    });
}

int tn_stokes_create(tn_shell* shell, int velocity_level, int precision, const void* k_nodal_dev,
                     const void* k_cell_dev, int bc_cmb, int bc_surface, tn_operator** out)
{
    return guarded([&] {
        need(shell && out, "NULL argument");
        auto s  = std::make_unique<tn::StokesOp>();
        auto sh = shell->impl.get();
        init_coupling(*s, sh, velocity_level, precision, bc_cmb, bc_surface);
        init_edd(s->A, sh, velocity_level, precision, k_nodal_dev, k_cell_dev, bc_cmb, bc_surface, 0);
        init_coupling(s->BT, sh, velocity_level, precision, bc_cmb, bc_surface);
        init_coupling(s->B, sh, velocity_level, precision, bc_cmb, bc_surface);
        auto o = new tn_operator;
        o->op  = std::move(s);
        *out   = o;
    });
}

void tn_operator_destroy(tn_operator* op) { delete op; }

int tn_operator_set_modes(tn_operator* op, int apply_mode, int comm_mode)
{
    return guarded([&] {
        need(op, "NULL operator");
        need(apply_mode == TN_REPLACE || apply_mode == TN_ADD, "invalid apply mode");
        need(comm_mode == TN_SKIP_COMMUNICATION || comm_mode == TN_COMMUNICATE_ADDITIVELY, "invalid comm mode");
        if (dynamic_cast<tn::StokesOp*>(op->op.get()) && apply_mode != TN_REPLACE)
            throw tn::Error(tn::kErrUnsupported, "the Stokes block operator applies in Replace mode only");
        op->op->apply_mode = apply_mode;
        op->op->comm_mode  = comm_mode;
    });
}

int tn_operator_set_diagonal(tn_operator* op, int diagonal)
{
    return guarded([&] {
        need(op, "NULL operator");
        as_edd(op)->diagonal = diagonal != 0;
    });
}

int tn_operator_set_boundary_conditions(tn_operator* op, int bc_cmb, int bc_surface)
{
    return guarded([&] {
        need(op, "NULL operator");
        check_bcs(bc_cmb, bc_surface);
        op->op->bc_cmb  = bc_cmb;
        op->op->bc_surf = bc_surface;
        if (auto* s = dynamic_cast<tn::StokesOp*>(op->op.get())) {
            s->A.bc_cmb = s->B.bc_cmb = s->BT.bc_cmb = bc_cmb;
            s->A.bc_surf = s->B.bc_surf = s->BT.bc_surf = bc_surface;
            s->A.prepare_penalty(nullptr);
        }
        if (auto* e = dynamic_cast<tn::EpsDivDivOp*>(op->op.get())) e->prepare_penalty(nullptr);
    });
}

int tn_operator_set_tile(tn_operator* op, int tile_y, int chunk_x)
{
    return guarded([&] {
        need(op, "NULL operator");
        auto* e = as_edd(op);
        need(tile_y >= 0 && tile_y <= (e->precision == TN_F64 ? 7 : 11) && chunk_x >= 0 && chunk_x <= 64,
             "tile out of range");
        e->tile_y  = tile_y;
        e->chunk_x = chunk_x;
    });
}

int tn_operator_components(const tn_operator* op, int* src_components, int* dst_components)
{
    return guarded([&] {
        need(op && src_components && dst_components, "NULL argument");
        *src_components = op->op->src_components();
        *dst_components = op->op->dst_components();
    });
}

int tn_operator_apply(tn_operator* op, const void* const* src_dev, void* const* dst_dev, void* stream)
{
    return guarded([&] {
        need(op && src_dev && dst_dev, "NULL argument");
        for (int c = 0; c < op->op->src_components(); ++c) need(src_dev[c] != nullptr, "NULL source component");
        for (int c = 0; c < op->op->dst_components(); ++c) need(dst_dev[c] != nullptr, "NULL destination component");
        op->op->apply(const_cast<void* const*>(src_dev), dst_dev, as_stream(stream));
    });
}

int tn_kmass_lumped_diagonal(tn_shell* shell, int level, int precision, const void* k_dev, void* diag_dev,
                             void* stream)
{
    return guarded([&] {
        need(shell && k_dev && diag_dev, "NULL argument");
        precision_size(precision);
        const auto& L  = shell->impl->level(level);
        auto        st = as_stream(stream);
        int         rc;
        if (precision == TN_F64) {
            double* d = static_cast<double*>(diag_dev);
            tn::zero_components<double>(L.nodes(), 1, &d, st);
            rc = tn::kmass_lumped_add<double>(L.nl(), L.nr(), L.coords<double>(), L.radii<double>(),
                                              static_cast<const double*>(k_dev), d, st);
            if (!rc) rc = tn::interface_sum<double>(L.iface, L.nr(), 1, &d, st);
        } else {
            float* d = static_cast<float*>(diag_dev);
            tn::zero_components<float>(L.nodes(), 1, &d, st);
            rc = tn::kmass_lumped_add<float>(L.nl(), L.nr(), L.coords<float>(), L.radii<float>(),
                                             static_cast<const float*>(k_dev), d, st);
            if (!rc) rc = tn::interface_sum<float>(L.iface, L.nr(), 1, &d, st);
        }
        if (rc) throw tn::Error(tn::kErrCuda, "k-mass launch failed");
    });
}

int tn_vector_mass_apply(tn_shell* shell, int level, int precision, const void* const* src_dev, void* const* dst_dev,
                         void* stream)
{
    return guarded([&] {
        need(shell && src_dev && dst_dev, "NULL argument");
        precision_size(precision);
        const auto& L  = shell->impl->level(level);
        auto        st = as_stream(stream);
        int         rc;
        if (precision == TN_F64) {
            auto d = reinterpret_cast<double* const*>(dst_dev);
            tn::zero_components<double>(L.nodes(), 3, d, st);
            rc = tn::vector_mass_add<double>(L.nl(), L.nr(), L.coords<double>(), L.radii<double>(),
                                             reinterpret_cast<const double* const*>(src_dev), d, st);
            if (!rc) rc = tn::interface_sum<double>(L.iface, L.nr(), 3, d, st);
        } else {
            auto d = reinterpret_cast<float* const*>(dst_dev);
            tn::zero_components<float>(L.nodes(), 3, d, st);
            rc = tn::vector_mass_add<float>(L.nl(), L.nr(), L.coords<float>(), L.radii<float>(),
                                            reinterpret_cast<const float* const*>(src_dev), d, st);
            if (!rc) rc = tn::interface_sum<float>(L.iface, L.nr(), 3, d, st);
        }
        if (rc) throw tn::Error(tn::kErrCuda, "vector mass launch failed");
    });
}

int tn_prolongate_add(tn_shell* shell, int fine_level, int precision, int ncomp, const void* const* coarse_dev,
                      void* const* fine_dev, void* stream)
{
    return guarded([&] {
        need(shell && coarse_dev && fine_dev, "NULL argument");
        need(ncomp >= 1 && ncomp <= 4, "ncomp must be 1..4");
        need(fine_level >= 1, "fine level needs a coarser level");
        precision_size(precision);
        const auto& L = shell->impl->level(fine_level);
        int         rc;
        if (precision == TN_F64)
            rc = tn::prolongate_add<double>(L.nl(), L.nr(), ncomp, reinterpret_cast<const double* const*>(coarse_dev),
                                            reinterpret_cast<double* const*>(fine_dev), as_stream(stream));
        else
            rc = tn::prolongate_add<float>(L.nl(), L.nr(), ncomp, reinterpret_cast<const float* const*>(coarse_dev),
                                           reinterpret_cast<float* const*>(fine_dev), as_stream(stream));
        if (rc) throw tn::Error(tn::kErrCuda, "prolongation launch failed");
    });
}

int tn_prolongate_linear_add(tn_shell* shell, int fine_level, int precision, int ncomp, const void* const* coarse_dev,
                             void* const* fine_dev, void* stream)
{
    return guarded([&] {
        need(shell && coarse_dev && fine_dev, "NULL argument");
        need(ncomp >= 1 && ncomp <= 4, "ncomp must be 1..4");
        need(fine_level >= 1, "fine level needs a coarser level");
        const auto& L  = shell->impl->level(fine_level);
        const int   rc = dispatch_prec(precision, [&](auto t) {
            using T = decltype(t);
            return tn::prolongate_linear_add<T>(L.nl(), L.nr(), ncomp, L.linear_weights<T>(as_stream(stream)),
                                                reinterpret_cast<const T* const*>(coarse_dev),
                                                reinterpret_cast<T* const*>(fine_dev), as_stream(stream));
        });
        if (rc) throw tn::Error(tn::kErrCuda, "prolongation launch failed");
    });
}

int tn_restrict_linear(tn_shell* shell, int fine_level, int precision, int ncomp, const void* const* fine_dev,
                       void* const* coarse_dev, void* stream)
{
    return guarded([&] {
        need(shell && coarse_dev && fine_dev, "NULL argument");
        need(ncomp >= 1 && ncomp <= 4, "ncomp must be 1..4");
        need(fine_level >= 1, "fine level needs a coarser level");
        const auto& L  = shell->impl->level(fine_level);
        const auto& Lc = shell->impl->level(fine_level - 1);
        const int   rc = dispatch_prec(precision, [&](auto t) {
            using T = decltype(t);
            auto c  = reinterpret_cast<T* const*>(coarse_dev);
            int  r  = tn::restrict_linear_owned<T>(L.nl(), L.nr(), ncomp, L.owned_lat.as<uint8_t>(),
                                                 L.linear_weights<T>(as_stream(stream)),
                                                 reinterpret_cast<const T* const*>(fine_dev), c, as_stream(stream));
            return r ? r : tn::interface_sum<T>(Lc.iface, Lc.nr(), ncomp, c, as_stream(stream));
        });
        if (rc) throw tn::Error(tn::kErrCuda, "restriction launch failed");
    });
}

int tn_restrict(tn_shell* shell, int fine_level, int precision, int ncomp, const void* const* fine_dev,
                void* const* coarse_dev, void* stream)
{
    return guarded([&] {
        need(shell && coarse_dev && fine_dev, "NULL argument");
        need(ncomp >= 1 && ncomp <= 4, "ncomp must be 1..4");
        need(fine_level >= 1, "fine level needs a coarser level");
        precision_size(precision);
        const auto& L  = shell->impl->level(fine_level);
        const auto& Lc = shell->impl->level(fine_level - 1);
        int         rc;
        if (precision == TN_F64) {
            auto c = reinterpret_cast<double* const*>(coarse_dev);
            rc     = tn::restrict_owned<double>(L.nl(), L.nr(), ncomp, L.owned_lat.as<uint8_t>(),
                                            reinterpret_cast<const double* const*>(fine_dev), c, as_stream(stream));
            if (!rc) rc = tn::interface_sum<double>(Lc.iface, Lc.nr(), ncomp, c, as_stream(stream));
        } else {
            auto c = reinterpret_cast<float* const*>(coarse_dev);
            rc     = tn::restrict_owned<float>(L.nl(), L.nr(), ncomp, L.owned_lat.as<uint8_t>(),
                                           reinterpret_cast<const float* const*>(fine_dev), c, as_stream(stream));
            if (!rc) rc = tn::interface_sum<float>(Lc.iface, Lc.nr(), ncomp, c, as_stream(stream));
        }
        if (rc) throw tn::Error(tn::kErrCuda, "restriction launch failed");
    });
}

int tn_interface_sum(tn_shell* shell, int level, int precision, int ncomp, void* const* comps_dev, void* stream)
{
    return guarded([&] {
        need(shell && comps_dev, "NULL argument");
        need(ncomp >= 1 && ncomp <= 4, "ncomp must be 1..4");
        precision_size(precision);
        const auto& L = shell->impl->level(level);
        int         rc;
        if (precision == TN_F64)
            rc = tn::interface_sum<double>(L.iface, L.nr(), ncomp, reinterpret_cast<double* const*>(comps_dev),
                                           as_stream(stream));
        else
            rc = tn::interface_sum<float>(L.iface, L.nr(), ncomp, reinterpret_cast<float* const*>(comps_dev),
                                          as_stream(stream));
        if (rc) throw tn::Error(tn::kErrCuda, "interface sum launch failed");
    });
}

int tn_vec_lincomb(tn_shell* shell, int level, int precision, int ncomp, void* const* y_dev, double c0, int nterms,
                   const double* c, const void* const* x0_dev, const void* const* x1_dev, const void* const* x2_dev,
                   void* stream)
{
    return guarded([&] {
        need(shell && y_dev, "NULL argument");
        need(ncomp >= 1 && ncomp <= 4 && nterms >= 0 && nterms <= 3, "bad ncomp / nterms");
        need(nterms == 0 || c != nullptr, "coefficients missing");
        precision_size(precision);
        const auto&   L = shell->impl->level(level);
        const int64_t n = L.nodes();
        int           rc;
        if (precision == TN_F64) {
            double cc[3] = {nterms > 0 ? c[0] : 0, nterms > 1 ? c[1] : 0, nterms > 2 ? c[2] : 0};
            rc           = tn::lincomb<double>(n, ncomp, reinterpret_cast<double* const*>(y_dev), c0, nterms, cc,
                                     reinterpret_cast<const double* const*>(x0_dev),
                                     reinterpret_cast<const double* const*>(x1_dev),
                                     reinterpret_cast<const double* const*>(x2_dev), as_stream(stream));
        } else {
            float cc[3] = {nterms > 0 ? float(c[0]) : 0.f, nterms > 1 ? float(c[1]) : 0.f, nterms > 2 ? float(c[2]) : 0.f};
            rc          = tn::lincomb<float>(n, ncomp, reinterpret_cast<float* const*>(y_dev), float(c0), nterms, cc,
                                    reinterpret_cast<const float* const*>(x0_dev),
                                    reinterpret_cast<const float* const*>(x1_dev),
                                    reinterpret_cast<const float* const*>(x2_dev), as_stream(stream));
        }
        if (rc) throw tn::Error(tn::kErrCuda, "lincomb launch failed");
    });
}

int tn_vec_dot(tn_shell* shell, int level, int precision, int ncomp, const void* const* a_dev,
               const void* const* b_dev, double* result, void* stream)
{
    return guarded([&] {
        need(shell && a_dev && b_dev && result, "NULL argument");
        need(ncomp >= 1 && ncomp <= 4, "ncomp must be 1..4");
        precision_size(precision);
        const auto& L   = shell->impl->level(level);
        double*     red = shell->impl->red.as<double>();
        int         rc;
        if (precision == TN_F64)
            rc = tn::masked_dot<double>(L.nodes(), L.nr(), ncomp, L.owned_lat.as<uint8_t>(),
                                        reinterpret_cast<const double* const*>(a_dev),
                                        reinterpret_cast<const double* const*>(b_dev), red, red + 8, as_stream(stream));
        else
            rc = tn::masked_dot<float>(L.nodes(), L.nr(), ncomp, L.owned_lat.as<uint8_t>(),
                                       reinterpret_cast<const float* const*>(a_dev),
                                       reinterpret_cast<const float* const*>(b_dev), red, red + 8, as_stream(stream));
        if (rc) throw tn::Error(tn::kErrCuda, "dot launch failed");
        tn::cuda_check(cudaMemcpyAsync(result, red, sizeof(double), cudaMemcpyDeviceToHost, as_stream(stream)),
                       "dot readback");
        tn::cuda_check(cudaStreamSynchronize(as_stream(stream)), "dot sync");
    });
}


/* ---- remaining VectorLike operations ----------------------------------- */
int tn_vec_invert(tn_shell* shell, int level, int precision, int ncomp, void* const* y_dev, void* stream)
{
    return guarded([&] {
        need(shell, "NULL shell");
        check_comps(ncomp, y_dev);
        const auto& L  = shell->impl->level(level);
        const int   rc = dispatch_prec(precision, [&](auto t) {
            using T = decltype(t);
            return tn::invert_inplace<T>(L.nodes(), ncomp, reinterpret_cast<T* const*>(y_dev), as_stream(stream));
        });
        if (rc) throw tn::Error(tn::kErrCuda, "invert launch failed");
    });
}

int tn_vec_scale(tn_shell* shell, int level, int precision, int ncomp, void* const* y_dev, const void* const* x_dev,
                 void* stream)
{
    return guarded([&] {
        need(shell && x_dev, "NULL argument");
        check_comps(ncomp, y_dev);
        const auto& L  = shell->impl->level(level);
        const int   rc = dispatch_prec(precision, [&](auto t) {
            using T = decltype(t);
            return tn::scale_inplace<T>(L.nodes(), ncomp, reinterpret_cast<T* const*>(y_dev),
                                        reinterpret_cast<const T* const*>(x_dev), as_stream(stream));
        });
        if (rc) throw tn::Error(tn::kErrCuda, "scale launch failed");
    });
}

int tn_vec_max_abs(tn_shell* shell, int level, int precision, int ncomp, const void* const* a_dev, double* result,
                   void* stream)
{
    return guarded([&] {
        need(shell && result, "NULL argument");
        max_abs_nan(shell, level, precision, ncomp, a_dev, result, nullptr, stream);
    });
}

int tn_vec_has_nan_or_inf(tn_shell* shell, int level, int precision, int ncomp, const void* const* a_dev, int* result,
                          void* stream)
{
    return guarded([&] {
        need(shell && result, "NULL argument");
        max_abs_nan(shell, level, precision, ncomp, a_dev, nullptr, result, stream);
    });
}

int tn_vec_swap(tn_shell* shell, int level, int precision, int ncomp, void* const* a_dev, void* const* b_dev,
                void* stream)
{
    return guarded([&] {
        need(shell && b_dev, "NULL argument");
        check_comps(ncomp, a_dev);
        const auto& L  = shell->impl->level(level);
        const int   rc = dispatch_prec(precision, [&](auto t) {
            using T = decltype(t);
            return tn::swap_vectors<T>(L.nodes(), ncomp, reinterpret_cast<T* const*>(a_dev),
                                       reinterpret_cast<T* const*>(b_dev), as_stream(stream));
        });
        if (rc) throw tn::Error(tn::kErrCuda, "swap launch failed");
    });
}

int tn_vec_cast(int64_t n, int direction, const void* in_dev, void* out_dev, void* stream)
{
    return guarded([&] {
        need(n >= 0 && (n == 0 || (in_dev && out_dev)), "bad arguments");
        precision_size(direction);
        if (n == 0) return;
        const int rc = direction == TN_F64
                           ? tn::convert_f64_to_f32(n, static_cast<const double*>(in_dev), static_cast<float*>(out_dev),
                                                    as_stream(stream))
                           : tn::convert_f32_to_f64(n, static_cast<const float*>(in_dev), static_cast<double*>(out_dev),
                                                    as_stream(stream));
        if (rc) throw tn::Error(tn::kErrCuda, "cast launch failed");
    });
}

/* ---- boundary treatment of right-hand sides ----------------------------- */
int tn_vec_assign_masked(tn_shell* shell, int level, int precision, int ncomp, void* const* v_dev, int flag,
                         double value, void* stream)
{
    return guarded([&] {
        need(shell, "NULL shell");
        check_comps(ncomp, v_dev);
        need(flag >= 0 && flag < 256, "flag must be a ShellBoundaryFlag value");
        const auto& L  = shell->impl->level(level);
        const int   rc = dispatch_prec(precision, [&](auto t) {
            using T = decltype(t);
            return tn::assign_masked<T>(L.nodes(), L.nr(), ncomp, reinterpret_cast<T* const*>(v_dev), flag,
                                        static_cast<T>(value), as_stream(stream));
        });
        if (rc) throw tn::Error(tn::kErrCuda, "assign launch failed");
    });
}

int tn_vec_rotate_normal_tangential(tn_shell* shell, int level, int precision, void* const* v_dev, int flag,
                                    int direction, void* stream)
{
    return guarded([&] {
        need(direction == 0 || direction == 1, "direction must be 0 or 1");
        rotate(shell, level, precision, v_dev, flag, direction, stream);
    });
}

int tn_vec_freeslip_project(tn_shell* shell, int level, int precision, void* const* v_dev, int flag, void* stream)
{
    return guarded([&] { rotate(shell, level, precision, v_dev, flag, 2, stream); });
}

int tn_stokes_rhs_enforce(tn_shell* shell, int level, int precision, int bc_cmb, int bc_surface, void* const* u_dev,
                          void* stream)
{
    return guarded([&] {
        need(shell, "NULL shell");
        check_bcs(bc_cmb, bc_surface);
        check_comps(3, u_dev);
        const auto& L     = shell->impl->level(level);
        const int   fdir  = shell_boundary_flag(bc_cmb, bc_surface, TN_DIRICHLET);
        const int   ffs   = shell_boundary_flag(bc_cmb, bc_surface, TN_FREESLIP);
        const int   rc    = dispatch_prec(precision, [&](auto t) {
            using T = decltype(t);
            auto* v = reinterpret_cast<T* const*>(u_dev);
            if (tn::assign_masked<T>(L.nodes(), L.nr(), 3, v, fdir, T(0), as_stream(stream)) != 0) return -1;
            return tn::rotate_normal_tangential<T>(L.nodes(), L.nr(), L.coords<T>(), v, ffs, 2, as_stream(stream));
        });
        if (rc) throw tn::Error(tn::kErrCuda, "right-hand-side launch failed");
    });
}

/* ---- stored matrices and Galerkin coarse operators ---------------------- */
int tn_operator_set_stored_matrix_mode(tn_operator* op, int mode, void* stream)
{
    return guarded([&] {
        need(op != nullptr, "NULL operator");
        need(mode == TN_STORED_OFF || mode == TN_STORED_FULL, "mode must be TN_STORED_OFF or TN_STORED_FULL");
        auto* e = as_edd(op);
        if (mode == TN_STORED_OFF) {
            need(e->k.get() != nullptr, "the operator has no coefficient for the matrix-free mode");
            e->stored = false;
            return;
        }
        e->set_stored_matrices_from_coefficient(as_stream(stream));
        tn::cuda_check(cudaStreamSynchronize(as_stream(stream)), "synchronize");
    });
}

int tn_gca_mark_elements(tn_shell* shell, int level, int level_range, const double* k_dev, uint8_t* marks_dev,
                         void* stream)
{
    return guarded([&] {
        need(shell && k_dev && marks_dev, "NULL argument");
        const auto& L = shell->impl->level(level);
        need(level_range >= 0 && level - level_range >= 0, "level_range must lead to a level of the shell");
        const auto& Lc = shell->impl->level(level - level_range);
        tn::cuda_check(cudaMemsetAsync(marks_dev, 0, static_cast<size_t>(Lc.cells()), as_stream(stream)),
                       "clear marks");
        if (tn::gca_mark_elements(L.nl(), L.nr(), k_dev, level_range, marks_dev, as_stream(stream)) != 0)
            throw tn::Error(tn::kErrCuda, "marking launch failed");
    });
}

int tn_operator_set_selective_matrices(tn_operator* op, int level_range, const uint8_t* marks_dev, void* stream)
{
    return guarded([&] {
        need(op && marks_dev, "NULL argument");
        as_edd(op)->set_selective(marks_dev, level_range, as_stream(stream));
    });
}

int tn_operator_stored_cells(tn_operator* op, int64_t* stored_cells, int64_t* bytes)
{
    return guarded([&] {
        need(op && stored_cells && bytes, "NULL argument");
        const auto* e = as_edd(op);
        *stored_cells = e->selective ? e->sel_count : (e->stored ? e->lvl().cells() : 0);
        *bytes = static_cast<int64_t>(e->mats.size() + e->sel_delta.size() + e->baked64.size() + e->baked32.size() +
                                      e->sel_cells.size() + e->sel_slot.size());
    });
}

int tn_gca_build(tn_operator* fine, tn_operator* coarse, void* stream)
{
    return tn_gca_build_interpolated(fine, coarse, TN_TRANSFER_CONSTANT, 1, stream);
}

int tn_gca_build_interpolated(tn_operator* fine, tn_operator* coarse, int interpolation, int tensor_cores,
                              void* stream)
{
    return guarded([&] {
        need(fine && coarse, "NULL operator");
        need(interpolation == TN_TRANSFER_CONSTANT || interpolation == TN_TRANSFER_LINEAR, "unknown interpolation");
        tn::gca_coarsen(*as_edd(fine), *as_edd(coarse), as_stream(stream), interpolation == TN_TRANSFER_LINEAR,
                        tensor_cores != 0);
        tn::cuda_check(cudaStreamSynchronize(as_stream(stream)), "synchronize");
    });
}

int tn_operator_copy_local_matrices(tn_operator* op, double* mats_host)
{
    return guarded([&] {
        need(op && mats_host, "NULL argument");
        unpack_matrices(*as_edd(op), mats_host);
    });
}

int tn_vec_alloc(tn_shell* shell, int level, int precision, int ncomp, void** comps_out)
{
    return guarded([&] {
        need(shell && comps_out, "NULL argument");
        need(ncomp >= 1 && ncomp <= 4, "ncomp must be 1..4");
        const size_t esz = precision_size(precision);
        const auto&  L   = shell->impl->level(level);
        // padded to 256 bytes so that 16-byte-rounded bulk reads stay inside the allocation
        const size_t bytes = (esz * static_cast<size_t>(L.nodes()) + 255) / 256 * 256;
        for (int c = 0; c < ncomp; ++c) comps_out[c] = nullptr;
        try {
            for (int c = 0; c < ncomp; ++c) {
                if (cudaMalloc(&comps_out[c], bytes) != cudaSuccess) {
                    cudaGetLastError();
                    comps_out[c] = nullptr;
                    throw tn::Error(tn::kErrAlloc, "cudaMalloc of " + std::to_string(bytes) + " bytes failed");
                }
                tn::cuda_check(cudaMemset(comps_out[c], 0, bytes), "zero vector");
            }
        } catch (...) {
            for (int c = 0; c < ncomp; ++c)
                if (comps_out[c]) cudaFree(comps_out[c]);
            for (int c = 0; c < ncomp; ++c) comps_out[c] = nullptr;
            throw;
        }
    });
}

void tn_vec_free(int ncomp, void* const* comps)
{
    if (!comps) return;
    for (int c = 0; c < ncomp; ++c)
        if (comps[c]) cudaFree(comps[c]);
}

int tn_sync(void* stream)
{
    return guarded([&] { tn::cuda_check(cudaStreamSynchronize(as_stream(stream)), "stream synchronize"); });
}

int tn_vec_random(tn_shell* shell, int level, int precision, int ncomp, uint64_t seed, void* const* comps_dev,
                  void* stream)
{
    return guarded([&] {
        need(shell && comps_dev, "NULL argument");
        need(ncomp >= 1 && ncomp <= 4, "ncomp must be 1..4");
        precision_size(precision);
        const auto& L = shell->impl->level(level);
        int         rc;
        if (precision == TN_F64)
            rc = tn::random_fill<double>(L.nodes(), ncomp, reinterpret_cast<double* const*>(comps_dev), L.nr(),
                                         L.canon_lat.as<int32_t>(), seed, as_stream(stream));
        else
            rc = tn::random_fill<float>(L.nodes(), ncomp, reinterpret_cast<float* const*>(comps_dev), L.nr(),
                                        L.canon_lat.as<int32_t>(), seed, as_stream(stream));
        if (rc) throw tn::Error(tn::kErrCuda, "random fill launch failed");
    });
}

/* ---- solvers ------------------------------------------------------------ */
void tn_solver_options_default(tn_solver_options* o)
{
    if (!o) return;
    o->restart                   = 30;
    o->max_iterations            = 300;
    o->relative_tolerance        = 1e-8;
    o->absolute_tolerance        = 1e-12;
    o->chebyshev_order           = 2;
    o->chebyshev_iterations      = 2;
    o->power_iterations          = 10;
    o->num_vcycles               = 1;
    o->coarse_max_iterations     = 50;
    o->coarse_relative_tolerance = 1e-6;
    o->coarse_absolute_tolerance = 1e-16;
    o->gca                       = 1;
    o->mixed_precision           = 0;
    o->seed                      = 12345;
    o->normalize_pressure        = 1;
    o->project_pressure_mean     = 0;
    o->cuda_graphs               = 1;
    o->smoother                  = TN_SMOOTHER_CHEBYSHEV;
    o->jacobi_omega              = 1.0;
    o->coarse_solver             = TN_COARSE_PCG;
    o->transfer                  = TN_TRANSFER_CONSTANT;
}

int tn_stokes_solver_create(tn_shell* shell, int velocity_level, const double* eta_nodal_dev,
                            const double* eta_cell_dev, const double* k_schur_dev, int bc_cmb, int bc_surface,
                            const tn_solver_options* opts, void* stream, tn_solver** out)
{
    return guarded([&] {
        need(shell && out, "NULL argument");
        check_bcs(bc_cmb, bc_surface);
        tn_solver_options o;
        tn_solver_options_default(&o);
        if (opts) o = *opts;
        tn::StokesOptions so;
        so.restart  = o.restart;
        so.max_iter = o.max_iterations;
        so.rtol     = o.relative_tolerance;
        so.atol     = o.absolute_tolerance;
        so.mg       = mg_options(o);
        so.normalize_pressure    = o.normalize_pressure != 0;
        so.project_pressure_mean = o.project_pressure_mean != 0;
        so.use_graphs            = o.cuda_graphs != 0;
        auto s      = std::make_unique<tn_solver>();
        s->shell    = shell;
        s->stokes   = std::make_unique<tn::StokesSolver>(shell->impl.get(), velocity_level, eta_nodal_dev,
                                                       eta_cell_dev, k_schur_dev, bc_cmb, bc_surface, so,
                                                       as_stream(stream));
        *out = s.release();
    });
}

namespace {
int velocity_solver_create(tn_shell* shell, int level, const double* eta_nodal_dev, const double* eta_cell_dev,
                              int bc_cmb, int bc_surface, const tn_solver_options* opts, void* stream,
                           tn_solver** out, bool multigrid_only)
{
    return guarded([&] {
        need(shell && out, "NULL argument");
        check_bcs(bc_cmb, bc_surface);
        tn_solver_options o;
        tn_solver_options_default(&o);
        if (opts) o = *opts;
        tn::VelocitySolverOptions vo;
        vo.max_iter = o.max_iterations;
        vo.rtol     = o.relative_tolerance;
        vo.atol     = o.absolute_tolerance;
        vo.mg       = mg_options(o);
        vo.multigrid_only = multigrid_only;
        auto s      = std::make_unique<tn_solver>();
        s->shell    = shell;
        s->velocity = std::make_unique<tn::VelocitySolver>(shell->impl.get(), level, eta_nodal_dev, eta_cell_dev,
                                                           bc_cmb, bc_surface, vo, as_stream(stream));
        *out = s.release();
    });
}

}  // namespace

int tn_velocity_solver_create(tn_shell* shell, int level, const double* eta_nodal_dev, const double* eta_cell_dev,
                              int bc_cmb, int bc_surface, const tn_solver_options* opts, void* stream,
                              tn_solver** out)
{
    return velocity_solver_create(shell, level, eta_nodal_dev, eta_cell_dev, bc_cmb, bc_surface, opts, stream, out,
                                  false);
}

int tn_multigrid_solver_create(tn_shell* shell, int level, const double* eta_nodal_dev, const double* eta_cell_dev,
                               int bc_cmb, int bc_surface, const tn_solver_options* opts, void* stream,
                               tn_solver** out)
{
    return velocity_solver_create(shell, level, eta_nodal_dev, eta_cell_dev, bc_cmb, bc_surface, opts, stream, out,
                                  true);
}

void tn_solver_destroy(tn_solver* s) { delete s; }

int tn_solver_solve(tn_solver* s, double* const* x_dev, const double* const* b_dev, void* stream)
{
    int converged = 0;
    const int rc  = guarded([&] {
        need(s && x_dev && b_dev, "NULL argument");
        if (s->stokes) {
            const double* fu[3] = {b_dev[0], b_dev[1], b_dev[2]};
            double*       u[3]  = {x_dev[0], x_dev[1], x_dev[2]};
            converged           = s->stokes->solve(u, x_dev[3], fu, b_dev[3], as_stream(stream));
        } else {
            converged = s->velocity->solve(x_dev, b_dev, as_stream(stream));
        }
    });
    if (rc != TN_OK) return rc;
    if (!converged) {
        g_last_error = "the solver stopped before reaching its tolerance";
        return TN_ERR_NOT_CONVERGED;
    }
    return TN_OK;
}

int tn_solver_result(const tn_solver* s, int* iterations, double* relative_residual, int* converged)
{
    return guarded([&] {
        need(s != nullptr, "NULL solver");
        const int    it = s->stokes ? s->stokes->iterations : s->velocity->iterations;
        const double rr = s->stokes ? s->stokes->final_relres : s->velocity->final_relres;
        const bool   cv = s->stokes ? s->stokes->converged : s->velocity->converged;
        if (iterations) *iterations = it;
        if (relative_residual) *relative_residual = rr;
        if (converged) *converged = cv ? 1 : 0;
    });
}

int tn_solver_full_residual(const tn_solver* s, double* relative_residual)
{
    return guarded([&] {
        need(s && relative_residual, "NULL argument");
        *relative_residual = s->stokes ? s->stokes->full_relres : s->velocity->final_relres;
    });
}

int tn_solver_history(const tn_solver* s, double* history_host, int capacity, int* length)
{
    return guarded([&] {
        need(s && length, "NULL argument");
        const auto& h = s->stokes ? s->stokes->history : s->velocity->history;
        *length       = static_cast<int>(h.size());
        if (history_host)
            for (int i = 0; i < capacity && i < static_cast<int>(h.size()); ++i) history_host[i] = h[i];
    });
}

int tn_solver_precondition(tn_solver* s, const double* const* v_dev, double* const* z_dev, void* stream)
{
    return guarded([&] {
        need(s && v_dev && z_dev, "NULL argument");
        if (s->stokes)
            s->stokes->precondition_external(v_dev, z_dev, as_stream(stream));
        else
            s->velocity->precondition_external(v_dev, z_dev, as_stream(stream));
    });
}

int tn_solver_vcycle(tn_solver* s, int precision, void* const* x_dev, const void* const* b_dev, void* stream)
{
    return guarded([&] {
        need(s && x_dev && b_dev, "NULL argument");
        precision_size(precision);
        if (precision == TN_F64)
            s->mg().solve_external<double>(reinterpret_cast<double* const*>(x_dev),
                                           reinterpret_cast<const double* const*>(b_dev), as_stream(stream));
        else
            s->mg().solve_external<float>(reinterpret_cast<float* const*>(x_dev),
                                          reinterpret_cast<const float* const*>(b_dev), as_stream(stream));
        tn::cuda_check(cudaStreamSynchronize(as_stream(stream)), "synchronize");
    });
}

int tn_solver_level_lambda(tn_solver* s, int level, double* lambda_max)
{
    return guarded([&] {
        need(s && lambda_max, "NULL argument");
        need(level >= 1 && level <= s->mg().fine_level(), "level must be in 1..fine level");
        *lambda_max = s->mg().lambda(level);
    });
}

int tn_solver_inverse_diagonal(tn_solver* s, int level, double* const* out_dev, void* stream)
{
    return guarded([&] {
        need(s && out_dev, "NULL argument");
        need(level >= 1 && level <= s->mg().fine_level(), "level must be in 1..fine level");
        const auto& d = s->mg().inv_diag(level);
        for (int c = 0; c < 3; ++c)
            tn::cuda_check(cudaMemcpyAsync(out_dev[c], d.comp(0, c), sizeof(double) * d.d.seg[0].n,
                                           cudaMemcpyDeviceToDevice, as_stream(stream)),
                           "copy");
        tn::cuda_check(cudaStreamSynchronize(as_stream(stream)), "synchronize");
    });
}

int tn_solver_coarse_stats(tn_solver* s, double* stats3)
{
    return guarded([&] {
        need(s && stats3, "NULL argument");
        s->mg().coarse_stats(stats3, nullptr);
    });
}

int tn_epsdivdiv_vjp(tn_operator* op, const void* const* u_dev, const void* const* lambda_dev,
                     void* grad_logeta_cell_dev, void* const* grad_u_dev, void* stream)
{
    return guarded([&] {
        need(op && u_dev && lambda_dev && grad_logeta_cell_dev, "NULL argument");
        auto* e = as_edd(op);
        if (e->precision == TN_F64)
            e->vjp_logeta<double>(reinterpret_cast<const double* const*>(u_dev),
                                  reinterpret_cast<const double* const*>(lambda_dev),
                                  static_cast<double*>(grad_logeta_cell_dev), as_stream(stream));
        else
            e->vjp_logeta<float>(reinterpret_cast<const float* const*>(u_dev),
                                 reinterpret_cast<const float* const*>(lambda_dev),
                                 static_cast<float*>(grad_logeta_cell_dev), as_stream(stream));
        if (grad_u_dev) {
            // A^T lambda = A lambda, Replace
            const int am = e->apply_mode;
            e->apply_mode = 0;
            try {
                e->apply(const_cast<void* const*>(lambda_dev), grad_u_dev, as_stream(stream));
            } catch (...) {
                e->apply_mode = am;
                throw;
            }
            e->apply_mode = am;
        }
    });
}

int tn_stokes_misfit_gradient(tn_solver* s, const double* const* x_dev, const double* const* u_obs_dev,
                              double* grad_logeta_cell_dev, double* const* lambda_dev, void* stream)
{
    int       converged = 0;
    const int rc        = guarded([&] {
        need(s && x_dev && u_obs_dev && grad_logeta_cell_dev, "NULL argument");
        need(s->stokes != nullptr, "not a Stokes solver");
        converged = s->stokes->misfit_gradient(x_dev, u_obs_dev, grad_logeta_cell_dev, lambda_dev, as_stream(stream));
    });
    if (rc != TN_OK) return rc;
    if (!converged) {
        g_last_error = "the adjoint solve stopped before reaching its tolerance";
        return TN_ERR_NOT_CONVERGED;
    }
    return TN_OK;
}

int tn_solver_level_matrices(tn_solver* s, int level, double* mats_host)
{
    return guarded([&] {
        need(s && mats_host, "NULL argument");
        need(level >= 0 && level < s->mg().fine_level(), "level must be a coarse level");
        unpack_matrices(s->mg().op64(level), mats_host);
    });
}

int tn_solver_level_storage(tn_solver* s, int level, int64_t* stored_cells, int64_t* bytes)
{
    return guarded([&] {
        need(s && stored_cells && bytes, "NULL argument");
        need(level >= 0 && level <= s->mg().fine_level(), "level out of range");
        const auto& e = s->mg().op64(level);
        *stored_cells = e.selective ? e.sel_count : (e.stored ? e.lvl().cells() : 0);
        *bytes = static_cast<int64_t>(e.mats.size() + e.sel_delta.size() + e.baked64.size() + e.baked32.size() +
                                      e.sel_cells.size() + e.sel_slot.size());
    });
}

}  // extern "C"

// Shell of an opaque handle and the thread's last-error message, for entry
// points defined in other translation units.
namespace tn {
Shell* shell_of(tn_shell* s) { return s ? s->impl.get() : nullptr; }
void   set_last_error(const std::string& message) { g_last_error = message; }
}  // namespace tn

extern "C" {

/* ---- XDMF output / checkpoint ------------------------------------------- */
int tn_xdmf_create(tn_shell* shell, int level, const char* directory, int geometry_bytes, tn_xdmf** out)
{
    return guarded([&] {
        need(shell && directory && out, "NULL argument");
        auto x  = std::make_unique<tn_xdmf>();
        x->impl = tn::xdmf_create(shell->impl.get(), level, directory, geometry_bytes);
        *out    = x.release();
    });
}

int tn_xdmf_add(tn_xdmf* x, const char* name, int precision, int ncomp, void* const* comps_dev, int output_bytes)
{
    return guarded([&] {
        need(x && name && comps_dev, "NULL argument");
        tn::xdmf_add(x->impl, name, precision, ncomp, comps_dev, output_bytes);
    });
}

int tn_xdmf_write(tn_xdmf* x, void* stream)
{
    return guarded([&] {
        need(x != nullptr, "NULL argument");
        tn::cuda_check(cudaStreamSynchronize(as_stream(stream)), "synchronize");
        tn::xdmf_write(x->impl);
    });
}

void tn_xdmf_destroy(tn_xdmf* x) { delete x; }

int tn_xdmf_read(tn_shell* shell, int level, const char* directory, const char* name, int step, int precision,
                 int ncomp, void* const* comps_dev)
{
    return guarded([&] {
        need(shell && directory && name && comps_dev, "NULL argument");
        need(ncomp >= 1 && ncomp <= 3, "ncomp must be 1..3");
        precision_size(precision);
        tn::xdmf_read(shell->impl.get(), level, directory, name, step, precision, ncomp, comps_dev);
    });
}

}  // extern "C"
