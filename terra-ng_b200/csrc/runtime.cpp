// Host runtime: device mesh construction and operator dispatch.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>

#include <type_traits>

#include "tn_boundary.hpp"
#include "tn_runtime.hpp"

namespace tn {

namespace {
std::atomic<uint64_t> g_launches{0};
}
void     note_launch(int kernels) { g_launches.fetch_add(static_cast<uint64_t>(kernels), std::memory_order_relaxed); }
uint64_t launch_count() { return g_launches.load(std::memory_order_relaxed); }

int reduction_partials_size();

std::unique_ptr<Shell> make_shell(int lat_level, int rad_level, int num_levels, double r_min, double r_max)
{
    if (num_levels < 1) throw Error(kErrArg, "num_levels must be >= 1");
    if (lat_level - (num_levels - 1) < 0 || rad_level - (num_levels - 1) < 1)
        throw Error(kErrArg, "too many levels: the coarsest level needs lat_level >= 0 and rad_level >= 1");
    if (rad_level > 7) throw Error(kErrUnsupported, "at most 128 radial layers are supported");
    if (!(r_min > 0.0 && r_min < r_max)) throw Error(kErrArg, "need 0 < r_min < r_max");
    auto sh   = std::make_unique<Shell>();
    sh->r_min = r_min;
    sh->r_max = r_max;
    for (int l = 0; l < num_levels; ++l) {
        const int ll = lat_level - (num_levels - 1 - l);
        const int rl = rad_level - (num_levels - 1 - l);
        auto      dl = std::make_unique<DeviceLevel>();
        try {
            dl->host = make_shell_level(ll, rl, r_min, r_max);
        } catch (const std::invalid_argument& e) {
            throw Error(kErrArg, e.what());
        }
        const ShellLevel& h = dl->host;
        dl->coords64        = upload(h.coords);
        std::vector<float> c32(h.coords.begin(), h.coords.end());
        dl->coords32 = upload(c32);
        dl->radii64  = upload(h.radii);
        std::vector<float> r32(h.radii.begin(), h.radii.end());
        dl->radii32           = upload(r32);
        dl->owned_lat         = upload(h.owned_lat);
        dl->dup_offset        = upload(h.dup_offset);
        dl->dup_members       = upload(h.dup_members);
        {
            std::vector<int32_t> canon(h.owned_lat.size());
            for (size_t i = 0; i < canon.size(); ++i) canon[i] = static_cast<int32_t>(i);
            for (size_t c = 0; c + 1 < h.dup_offset.size(); ++c) {
                int32_t lo = h.dup_members[h.dup_offset[c]];
                for (int32_t m = h.dup_offset[c]; m < h.dup_offset[c + 1]; ++m) lo = std::min(lo, h.dup_members[m]);
                for (int32_t m = h.dup_offset[c]; m < h.dup_offset[c + 1]; ++m) canon[h.dup_members[m]] = lo;
            }
            dl->canon_lat = upload(canon);
        }
        if (h.nl > 1) {
            const size_t ncol = static_cast<size_t>(10) * (h.nl - 1) * (h.nl - 1) * 20;
            dl->colgeo64.alloc(ncol * sizeof(double));
            dl->colgeo32.alloc(ncol * sizeof(float));
            if (column_geometry_table<double>(h.nl, dl->coords64.as<double>(), dl->colgeo64.as<double>(), nullptr) != 0 ||
                column_geometry_table<float>(h.nl, dl->coords32.as<float>(), dl->colgeo32.as<float>(), nullptr) != 0)
                throw Error(kErrCuda, "column geometry launch failed");
            cuda_check(cudaDeviceSynchronize(), "column geometry");
        }
        if (h.nr > 1) {
            dl->radgeo64.alloc(static_cast<size_t>(h.nr - 1) * 3 * sizeof(double));
            dl->radgeo32.alloc(static_cast<size_t>(h.nr - 1) * 3 * sizeof(float));
            if (radial_geometry_table<double>(h.nr, dl->radii64.as<double>(), dl->radgeo64.as<double>(), nullptr) != 0 ||
                radial_geometry_table<float>(h.nr, dl->radii32.as<float>(), dl->radgeo32.as<float>(), nullptr) != 0)
                throw Error(kErrCuda, "radial geometry launch failed");
            cuda_check(cudaDeviceSynchronize(), "radial geometry");
        }
        dl->iface.num_classes = static_cast<int>(h.dup_offset.size()) - 1;
        dl->iface.offset      = dl->dup_offset.as<int32_t>();
        dl->iface.members     = dl->dup_members.as<int32_t>();
        sh->levels.push_back(std::move(dl));
    }
    sh->err.alloc(sizeof(int));
    cuda_check(cudaMemset(sh->err.get(), 0, sizeof(int)), "memset err");
    sh->red.alloc(sizeof(double) * (reduction_partials_size() + 8));
    return sh;
}

template <>
const double* DeviceLevel::linear_weights<double>(cudaStream_t st) const
{
    if (linw64.get() == nullptr) {
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        cuda_check(cudaStreamIsCapturing(st, &cap), "capture status");
        if (cap != cudaStreamCaptureStatusNone)
            throw Error(kErrState, "linear-transfer weights must be built before stream capture");
        DevBuf w(sizeof(double) * 2 * static_cast<size_t>(nodes()));
        if (linear_transfer_weights(nl(), nr(), coords64.as<double>(), radii64.as<double>(), w.as<double>(), st) != 0)
            throw Error(kErrCuda, "linear-transfer weight launch failed");
        cuda_check(cudaStreamSynchronize(st), "linear-transfer weights");
        linw64 = std::move(w);
    }
    return linw64.as<double>();
}

template <>
const float* DeviceLevel::linear_weights<float>(cudaStream_t st) const
{
    if (linw32.get() == nullptr) {
        const double* w64 = linear_weights<double>(st);
        DevBuf        w(sizeof(float) * 2 * static_cast<size_t>(nodes()));
        if (convert_f64_to_f32(2 * nodes(), w64, w.as<float>(), st) != 0)
            throw Error(kErrCuda, "conversion launch failed");
        cuda_check(cudaStreamSynchronize(st), "linear-transfer weights");
        linw32 = std::move(w);
    }
    return linw32.as<float>();
}

template <typename T>
void zero_components(int64_t n, int ncomp, T* const* v, cudaStream_t st)
{
    for (int c = 0; c < ncomp; ++c) cuda_check(cudaMemsetAsync(v[c], 0, static_cast<size_t>(n) * sizeof(T), st), "zero");
}
template void zero_components<double>(int64_t, int, double* const*, cudaStream_t);
template void zero_components<float>(int64_t, int, float* const*, cudaStream_t);

namespace {
template <typename T>
void check_aligned(const void* p)
{
    if (reinterpret_cast<uintptr_t>(p) % sizeof(T) != 0)
        throw Error(kErrArg, "vector component pointers must be aligned to the element size");
}
template <typename T>
void iface(const DeviceLevel& L, int ncomp, T* const* v, cudaStream_t st)
{
    if (interface_sum<T>(L.iface, L.nr(), ncomp, v, st) != 0) throw Error(kErrCuda, "interface sum launch failed");
}
}  // namespace

int64_t EpsDivDivOp::mats_values() const
{
    return static_cast<int64_t>(gca_values_per_cell()) * (selective ? sel_count : lvl().cells());
}

void EpsDivDivOp::set_stored_matrices_from_coefficient(cudaStream_t st)
{
    const DeviceLevel& L = lvl();
    if (precision != 0) throw Error(kErrUnsupported, "stored matrices are assembled from an FP64 coefficient");
    if (k.get() == nullptr) throw Error(kErrState, "operator has no coefficient to assemble matrices from");
    selective = false;
    sel_built = false;
    mats.alloc(static_cast<size_t>(mats_values()) * sizeof(double));
    if (element_matrices(L.nl(), L.nr(), L.coords<double>(), L.radii<double>(), q0 ? nullptr : k.as<double>(),
                         q0 ? k.as<double>() : nullptr, mats.as<double>(), st) != 0)
        throw Error(kErrCuda, "element matrix assembly launch failed");
    stored        = true;
    baked_bc[0]   = -1;
    baked32_valid = false;
}

void EpsDivDivOp::set_selective(const uint8_t* marks_dev, int level_range, cudaStream_t st)
{
    const DeviceLevel& L = lvl();
    if (precision != 0 || k.get() == nullptr)
        throw Error(kErrUnsupported, "selective storage needs the FP64 coefficient of the on-the-fly operator");
    const int nl = L.nl(), nr = L.nr();
    if (level_range < 0 || ((nl - 1) >> level_range) < 1 || ((nr - 1) >> level_range) < 1 ||
        (((nl - 1) >> level_range) << level_range) != nl - 1 || (((nr - 1) >> level_range) << level_range) != nr - 1)
        throw Error(kErrArg, "level_range does not lead to a coarser level of this shell");
    const int nlc = ((nl - 1) >> level_range) + 1, nrc = ((nr - 1) >> level_range) + 1;
    std::vector<uint8_t> marks(static_cast<size_t>(10) * (nlc - 1) * (nlc - 1) * (nrc - 1));
    cuda_check(cudaMemcpyAsync(marks.data(), marks_dev, marks.size(), cudaMemcpyDeviceToHost, st), "copy marks");
    cuda_check(cudaStreamSynchronize(st), "copy marks");
    const int64_t        nc = L.cells();
    std::vector<int32_t> cells, slot(static_cast<size_t>(nc), -1);
    int64_t              c = 0;
    for (int d = 0; d < 10; ++d)
        for (int x = 0; x < nl - 1; ++x)
            for (int y = 0; y < nl - 1; ++y)
                for (int r = 0; r < nr - 1; ++r, ++c) {
                    const int64_t a = ((static_cast<int64_t>(d) * (nlc - 1) + (x >> level_range)) * (nlc - 1) +
                                       (y >> level_range)) *
                                          (nrc - 1) +
                                      (r >> level_range);
                    if (marks[static_cast<size_t>(a)]) {
                        slot[static_cast<size_t>(c)] = static_cast<int32_t>(cells.size());
                        cells.push_back(static_cast<int32_t>(c));
                    }
                }
    sel_cells       = upload(cells);
    sel_slot        = upload(slot);
    sel_count       = static_cast<int>(cells.size());
    sel_level_range = level_range;
    selective       = true;
    sel_built       = false;
    stored          = false;
    mats.release();
    sel_delta.release();
    baked64.release();
    baked32.release();
    baked_bc[0]   = -1;
    baked32_valid = false;
}

void EpsDivDivOp::finish_selective(cudaStream_t st)
{
    const DeviceLevel& L = lvl();
    if (!selective) throw Error(kErrState, "the operator has no selective storage");
    sel_delta.ensure(static_cast<size_t>(mats_values()) * sizeof(double));
    if (element_matrices(L.nl(), L.nr(), L.coords<double>(), L.radii<double>(), q0 ? nullptr : k.as<double>(),
                         q0 ? k.as<double>() : nullptr, sel_delta.as<double>(), st, sel_cells.as<int>(), sel_count,
                         mats.as<double>()) != 0)
        throw Error(kErrCuda, "correction matrix launch failed");
    sel_built     = true;
    baked_bc[0]   = -1;
    baked32_valid = false;
}

void EpsDivDivOp::effective_matrices(DevBuf& out, cudaStream_t st) const
{
    const DeviceLevel& L  = lvl();
    const int64_t      nc = L.cells();
    out.alloc(static_cast<size_t>(gca_values_per_cell()) * nc * sizeof(double));
    if (stored) {
        cuda_check(cudaMemcpyAsync(out.get(), mats.get(), out.size(), cudaMemcpyDeviceToDevice, st), "copy");
        return;
    }
    if (k.get() == nullptr || precision != 0) throw Error(kErrState, "no FP64 coefficient to assemble matrices from");
    if (element_matrices(L.nl(), L.nr(), L.coords<double>(), L.radii<double>(), q0 ? nullptr : k.as<double>(),
                         q0 ? k.as<double>() : nullptr, out.as<double>(), st) != 0)
        throw Error(kErrCuda, "element matrix assembly launch failed");
    if (selective && sel_built &&
        gca_scatter_slots(sel_count, sel_cells.as<int>(), mats.as<double>(), static_cast<int>(nc), out.as<double>(),
                          st) != 0)
        throw Error(kErrCuda, "scatter launch failed");
}

void EpsDivDivOp::materialize_full(cudaStream_t st)
{
    if (!selective) return;
    DevBuf full;
    effective_matrices(full, st);
    cuda_check(cudaStreamSynchronize(st), "materialize");
    mats      = std::move(full);
    selective = false;
    sel_built = false;
    sel_count = 0;
    sel_cells.release();
    sel_slot.release();
    sel_delta.release();
    baked64.release();
    baked32.release();
    stored        = true;
    baked_bc[0]   = -1;
    baked32_valid = false;
}

void EpsDivDivOp::prepare_fp32(cudaStream_t st)
{
    if (precision != 0) return;
    if (selective && k32.get() == nullptr) {
        const int64_t n = static_cast<int64_t>(k.size() / sizeof(double));
        DevBuf        b(sizeof(float) * static_cast<size_t>(n));
        if (convert_f64_to_f32(n, k.as<double>(), b.as<float>(), st) != 0)
            throw Error(kErrCuda, "conversion launch failed");
        k32 = std::move(b);
    }
    prepare_penalty(st);
    cuda_check(cudaStreamSynchronize(st), "prepare fp32");
}

void EpsDivDivOp::ensure_baked(bool need32, cudaStream_t st)
{
    const DeviceLevel& L   = lvl();
    const DevBuf&      src = selective ? sel_delta : mats;
    if (selective ? !sel_built : (!stored || mats.get() == nullptr))
        throw Error(kErrState, "stored matrix mode without matrices");
    const size_t nv = static_cast<size_t>(mats_values());
    if (nv == 0) return;
    if (baked_bc[0] != bc_cmb || baked_bc[1] != bc_surf || baked64.get() == nullptr) {
        if (baked64.get() == nullptr) baked64.alloc(nv * sizeof(double));
        cuda_check(cudaMemcpyAsync(baked64.get(), src.get(), nv * sizeof(double), cudaMemcpyDeviceToDevice, st),
                   "copy matrices");
        if (gca_bake_boundary(L.nl(), L.nr(), L.coords<double>(), L.radii<double>(), bc_cmb, bc_surf,
                              baked64.as<double>(), st, selective ? sel_cells.as<int>() : nullptr, sel_count) != 0)
            throw Error(kErrCuda, "boundary bake launch failed");
        baked_bc[0]   = bc_cmb;
        baked_bc[1]   = bc_surf;
        baked32_valid = false;
    }
    if (need32 && !baked32_valid) {
        if (baked32.get() == nullptr) baked32.alloc(nv * sizeof(float));
        if (gca_to_f32(static_cast<int64_t>(nv), baked64.as<double>(), baked32.as<float>(), st) != 0)
            throw Error(kErrCuda, "matrix conversion launch failed");
        baked32_valid = true;
    }
}

void gca_coarsen(const EpsDivDivOp& fine, EpsDivDivOp& coarse, cudaStream_t st, bool linear, bool tensor_cores)
{
    if (fine.shell != coarse.shell || coarse.level != fine.level - 1)
        throw Error(kErrArg, "GCA needs operators on consecutive levels of one shell");
    const DeviceLevel& Lf       = fine.lvl();
    const bool         fine_sel = fine.selective && fine.sel_built;
    if (!fine.stored && !fine_sel && (fine.precision != 0 || fine.k.get() == nullptr))
        throw Error(kErrUnsupported, "GCA needs an FP64 fine coefficient or stored fine matrices");
    GcaSlots sl;
    if (fine_sel) {
        // TwoGridGCA reads get_local_matrix of the fine children, which a selective store only has for the
        // children of marked cells (gca.hpp:157-163, epsilon_divdiv_kerngen.hpp:546-562)
        if (!coarse.selective || coarse.sel_level_range != fine.sel_level_range - 1)
            throw Error(kErrUnsupported,
                        "a selectively stored fine operator can only be coarsened into a selective operator "
                        "with the same marks");
        sl.fine_slot   = fine.sel_slot.as<int>();
        sl.fine_stride = fine.sel_count;
    }
    if (coarse.selective) {
        sl.cells  = coarse.sel_cells.as<int>();
        sl.nslots = coarse.sel_count;
    }
    sl.err = coarse.shell->err_word();
    coarse.mats.ensure(static_cast<size_t>(coarse.mats_values()) * sizeof(double));
    const bool    on_the_fly = !fine.stored && !fine_sel;
    const double* kf         = (on_the_fly && !fine.q0) ? fine.k.as<double>() : nullptr;
    const double* kq0f       = (on_the_fly && fine.q0) ? fine.k.as<double>() : nullptr;
    const double* linw       = linear ? Lf.linear_weights<double>(st) : nullptr;
    if (gca_build(Lf.nl(), Lf.nr(), Lf.coords<double>(), Lf.radii<double>(), kf, kq0f,
                  on_the_fly ? nullptr : fine.mats.as<double>(), coarse.mats.as<double>(), st, linw, tensor_cores,
                  sl) != 0)
        throw Error(kErrCuda, "GCA build launch failed");
    if (coarse.selective) {
        coarse.finish_selective(st);
        return;
    }
    coarse.stored        = true;
    coarse.baked_bc[0]   = -1;
    coarse.baked32_valid = false;
}

void EpsDivDivOp::prepare_penalty(cudaStream_t st)
{
    if (!penalty_active() || pen_ready) return;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cuda_check(cudaStreamIsCapturing(st, &cap), "capture status");
    if (cap != cudaStreamCaptureStatusNone)
        throw Error(kErrState, "the free-slip null-space modes must be built before stream capture");
    const DeviceLevel& L = lvl();
    pen_scratch.alloc(sizeof(double) * (penalty_partials_size() + 8));
    double* ps = pen_scratch.as<double>();
    if (penalty_gram(L.nodes(), L.nr(), L.owned_lat.as<uint8_t>(), L.coords<double>(), L.radii<double>(), ps + 8, ps,
                     st) != 0)
        throw Error(kErrCuda, "null-space Gram launch failed");
    double g6[6];
    cuda_check(cudaMemcpyAsync(g6, ps, sizeof(g6), cudaMemcpyDeviceToHost, st), "Gram readback");
    cuda_check(cudaStreamSynchronize(st), "Gram sync");
    const double G[3][3] = {{g6[0], g6[1], g6[2]}, {g6[1], g6[3], g6[4]}, {g6[2], g6[4], g6[5]}};
    auto         inner   = [&](const double* a, const double* b) {
        double v = 0.0;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) v += a[i] * G[i][j] * b[j];
        return v;
    };
    // modified Gram-Schmidt with owned-node dots, then normalisation (epsilon_divdiv_kerngen.hpp:403-440), on the
    // coefficients of the modes in the raw basis
    double C[3][3] = {};
    for (int i = 0; i < 3; ++i) {
        double a[3] = {0.0, 0.0, 0.0};
        a[i]        = 1.0;
        for (int j = 0; j < i; ++j) {
            const double d = inner(a, C[j]);
            for (int q = 0; q < 3; ++q) a[q] -= d * C[j][q];
        }
        const double inv = 1.0 / std::sqrt(inner(a, a));
        for (int q = 0; q < 3; ++q) C[i][q] = a[q] * inv;
    }
    for (int i = 0; i < 3; ++i)
        for (int q = 0; q < 3; ++q) pen_coef.c[3 * i + q] = C[i][q];
    pen_ready = true;
}

template <typename T>
void EpsDivDivOp::add_penalty(const T* const* src, T* const* dst, cudaStream_t st)
{
    if (!penalty_active() || diagonal) return;
    prepare_penalty(st);
    const DeviceLevel& L  = lvl();
    double*            ps = pen_scratch.as<double>();
    if (penalty_apply<T>(L.nodes(), L.nr(), L.owned_lat.as<uint8_t>(), L.coords<T>(), L.radii<T>(), src, dst,
                         pen_coef, kPenaltyEpsilon, ps + 8, ps, st) != 0)
        throw Error(kErrCuda, "penalty launch failed");
}

template <typename T>
void EpsDivDivOp::vjp_logeta(const T* const* u, const T* const* lam, T* grad_cell, cudaStream_t st) const
{
    if (!q0 || k.get() == nullptr)
        throw Error(kErrUnsupported, "the log-viscosity gradient needs a per-cell (Q0) coefficient");
    if (stored) throw Error(kErrUnsupported, "the log-viscosity gradient needs the matrix-free operator");
    const DeviceLevel& L = lvl();
    VjpLaunch<T>       p;
    p.nl      = L.nl();
    p.nr      = L.nr();
    p.coords  = L.coords<T>();
    p.radii   = L.radii<T>();
    p.kq0     = k.as<T>();
    p.bc_cmb  = bc_cmb;
    p.bc_surf = bc_surf;
    p.grad    = grad_cell;
    for (int c = 0; c < 3; ++c) {
        p.u[c]   = u[c];
        p.lam[c] = lam[c];
    }
    if (epsdivdiv_vjp_logeta<T>(p, st) != 0) throw Error(kErrCuda, "vjp launch failed");
}
template void EpsDivDivOp::vjp_logeta<double>(const double* const*, const double* const*, double*, cudaStream_t) const;
template void EpsDivDivOp::vjp_logeta<float>(const float* const*, const float* const*, float*, cudaStream_t) const;

template <typename T>
void EpsDivDivOp::apply_t(const T* const* src, T* const* dst, cudaStream_t st)
{
    const DeviceLevel& L = lvl();
    for (int c = 0; c < 3; ++c) {
        check_aligned<T>(src[c]);
        check_aligned<T>(dst[c]);
    }
    if (stored) {
        if (apply_mode == 0) zero_components<T>(L.nodes(), 3, dst, st);
        if (diagonal) {
            if (!std::is_same<T, double>::value)
                throw Error(kErrUnsupported, "diagonal mode of a stored operator is FP64 only");
            if (gca_diag_add(L.nl(), L.nr(), L.coords<double>(), L.radii<double>(), bc_cmb, bc_surf,
                             mats.as<double>(), reinterpret_cast<const double* const*>(src),
                             reinterpret_cast<double* const*>(dst), st) != 0)
                throw Error(kErrCuda, "stored diagonal launch failed");
        } else {
            ensure_baked(std::is_same<T, float>::value, st);
            const T* m = std::is_same<T, float>::value ? static_cast<const T*>(baked32.get())
                                                       : static_cast<const T*>(baked64.get());
            if (gca_apply_add<T>(L.nl(), L.nr(), m, src, dst, st) != 0)
                throw Error(kErrCuda, "stored apply launch failed");
            add_penalty<T>(src, dst, st);
        }
        if (comm_mode == 1) iface<T>(L, 3, dst, st);
        return;
    }
    // matrix-free over every cell; a selective store adds its correction over the stored cells below
    const bool fp32_of_fp64 = std::is_same<T, float>::value && precision == 0;
    if (fp32_of_fp64 && (!selective || k32.get() == nullptr))
        throw Error(kErrState, "FP32 apply of an FP64 matrix-free operator needs prepare_fp32 (selective only)");
    const T*     kk = fp32_of_fp64 ? k32.as<T>() : k.as<T>();
    EddLaunch<T> p;
    p.nl     = L.nl();
    p.nr     = L.nr();
    p.coords = L.coords<T>();
    p.radii  = L.radii<T>();
    if (q0)
        p.kq0 = kk;
    else
        p.k = kk;
    for (int c = 0; c < 3; ++c) {
        p.src[c] = src[c];
        p.dst[c] = dst[c];
    }
    p.bc_cmb   = bc_cmb;
    p.bc_surf  = bc_surf;
    p.diagonal = diagonal;
    p.add      = apply_mode;
    p.tile_y   = tile_y;
    p.chunk_x  = chunk_x;
    p.err      = shell->err_word();
    const int rc = epsdivdiv_apply<T>(p, st);
    if (rc != 0) throw Error(kErrCuda, "epsdivdiv launch failed (" + std::to_string(rc) + ")");
    if (selective && sel_built && sel_count > 0) {
        if (diagonal) {
            if (!std::is_same<T, double>::value)
                throw Error(kErrUnsupported, "diagonal mode of a stored operator is FP64 only");
            if (gca_diag_add(L.nl(), L.nr(), L.coords<double>(), L.radii<double>(), bc_cmb, bc_surf,
                             sel_delta.as<double>(), reinterpret_cast<const double* const*>(src),
                             reinterpret_cast<double* const*>(dst), st, sel_cells.as<int>(), sel_count) != 0)
                throw Error(kErrCuda, "stored diagonal launch failed");
        } else {
            ensure_baked(std::is_same<T, float>::value, st);
            const T* m = std::is_same<T, float>::value ? static_cast<const T*>(baked32.get())
                                                       : static_cast<const T*>(baked64.get());
            if (gca_apply_add<T>(L.nl(), L.nr(), m, src, dst, st, sel_cells.as<int>(), sel_count) != 0)
                throw Error(kErrCuda, "stored apply launch failed");
        }
    }
    add_penalty<T>(src, dst, st);
    if (comm_mode == 1) iface<T>(L, 3, dst, st);
}
template void EpsDivDivOp::apply_t<double>(const double* const*, double* const*, cudaStream_t);
template void EpsDivDivOp::apply_t<float>(const float* const*, float* const*, cudaStream_t);

void EpsDivDivOp::apply(void* const* src, void* const* dst, cudaStream_t st)
{
    if (precision == 0)
        apply_t<double>(reinterpret_cast<const double* const*>(src), reinterpret_cast<double* const*>(dst), st);
    else
        apply_t<float>(reinterpret_cast<const float* const*>(src), reinterpret_cast<float* const*>(dst), st);
}

template <typename T>
void DivergenceOp::apply_t(const T* const* src, T* p, cudaStream_t st) const
{
    const DeviceLevel& L = lvl();
    if (level < 1) throw Error(kErrArg, "divergence needs a coarser pressure level");
    const DeviceLevel& Lc = shell->level(level - 1);
    if (apply_mode == 0) zero_components<T>(Lc.nodes(), 1, &p, st);
    CouplingLaunch<T> c;
    c.nl     = L.nl();
    c.nr     = L.nr();
    c.coords = L.coords<T>();
    c.colgeo = L.colgeo<T>();
    c.radgeo = L.radgeo<T>();
    c.radii  = L.radii<T>();
    c.bc_cmb = bc_cmb;
    c.bc_surf = bc_surf;
    for (int k = 0; k < 3; ++k) c.u[k] = src[k];
    c.p_out = p;
    const size_t need = sizeof(T) * 2 * static_cast<size_t>(L.cells());
    if (scratch.size() < need) scratch.alloc(need);
    c.wedge_scratch = scratch.as<T>();
    if (divergence_apply<T>(c, st) != 0) throw Error(kErrCuda, "divergence launch failed");
    if (comm_mode == 1) iface<T>(Lc, 1, &p, st);
}

void DivergenceOp::apply(void* const* src, void* const* dst, cudaStream_t st)
{
    if (precision == 0)
        apply_t<double>(reinterpret_cast<const double* const*>(src), static_cast<double*>(dst[0]), st);
    else
        apply_t<float>(reinterpret_cast<const float* const*>(src), static_cast<float*>(dst[0]), st);
}

template <typename T>
void GradientOp::apply_t(const T* p, T* const* dst, cudaStream_t st) const
{
    const DeviceLevel& L = lvl();
    if (level < 1) throw Error(kErrArg, "gradient needs a coarser pressure level");
    CouplingLaunch<T> c;
    c.nl      = L.nl();
    c.nr      = L.nr();
    c.coords  = L.coords<T>();
    c.colgeo  = L.colgeo<T>();
    c.radgeo  = L.radgeo<T>();
    c.radii   = L.radii<T>();
    c.add     = apply_mode == 1 ? 1 : 0;
    const size_t need = sizeof(T) * 2 * static_cast<size_t>(L.cells());
    if (scratch.size() < need) scratch.alloc(need);
    c.wedge_scratch = scratch.as<T>();
    c.bc_cmb  = bc_cmb;
    c.bc_surf = bc_surf;
    c.p_in    = p;
    for (int k = 0; k < 3; ++k) c.u_out[k] = dst[k];
    if (gradient_apply<T>(c, st) != 0) throw Error(kErrCuda, "gradient launch failed");
    if (comm_mode == 1) iface<T>(L, 3, dst, st);
}

void GradientOp::apply(void* const* src, void* const* dst, cudaStream_t st)
{
    if (precision == 0)
        apply_t<double>(static_cast<const double*>(src[0]), reinterpret_cast<double* const*>(dst), st);
    else
        apply_t<float>(static_cast<const float*>(src[0]), reinterpret_cast<float* const*>(dst), st);
}

// EpsDivDivStokes::apply_impl (epsilon_divdiv_stokes.hpp:55-84): A Replace +
// Skip into dst.u, B^T Add + communicate into dst.u (one interface sum for both),
// B Replace + communicate into dst.p. Always Replace, like the reference.
void StokesOp::apply(void* const* src, void* const* dst, cudaStream_t st)
{
    if (apply_mode != 0) throw Error(kErrUnsupported, "the Stokes block operator applies in Replace mode only");
    void* const su[3] = {src[0], src[1], src[2]};
    void* const du[3] = {dst[0], dst[1], dst[2]};
    void* const sp[1] = {src[3]};
    void* const dp[1] = {dst[3]};
    A.apply_mode      = 0;
    A.comm_mode       = 0;
    A.apply(su, du, st);
    BT.apply_mode = 1;
    BT.comm_mode  = comm_mode;
    BT.apply(sp, du, st);
    B.apply_mode = apply_mode;
    B.comm_mode  = comm_mode;
    B.apply(su, dp, st);
}

}  // namespace tn
