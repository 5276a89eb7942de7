// Host runtime: device mesh construction and operator dispatch.
#include <cstring>

#include "tn_runtime.hpp"

namespace tn {

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

template <typename T>
void EpsDivDivOp::apply_t(const T* const* src, T* const* dst, cudaStream_t st) const
{
    const DeviceLevel& L = lvl();
    EddLaunch<T>       p;
    p.nl     = L.nl();
    p.nr     = L.nr();
    p.coords = L.coords<T>();
    p.radii  = L.radii<T>();
    if (q0)
        p.kq0 = k.as<T>();
    else
        p.k = k.as<T>();
    for (int c = 0; c < 3; ++c) {
        p.src[c] = src[c];
        p.dst[c] = dst[c];
        check_aligned<T>(src[c]);
        check_aligned<T>(dst[c]);
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
    if (comm_mode == 1) iface<T>(L, 3, dst, st);
}

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
    c.radii  = L.radii<T>();
    c.bc_cmb = bc_cmb;
    c.bc_surf = bc_surf;
    for (int k = 0; k < 3; ++k) c.u[k] = src[k];
    c.p_out = p;
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
    if (apply_mode == 0) zero_components<T>(L.nodes(), 3, dst, st);
    CouplingLaunch<T> c;
    c.nl      = L.nl();
    c.nr      = L.nr();
    c.coords  = L.coords<T>();
    c.radii   = L.radii<T>();
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
