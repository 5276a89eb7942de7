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
void EpsDivDivOp::apply(const T* const* src, T* const* dst, cudaStream_t st, bool diag_override) const
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
        if ((reinterpret_cast<uintptr_t>(src[c]) % sizeof(T)) != 0 || (reinterpret_cast<uintptr_t>(dst[c]) % sizeof(T)) != 0)
            throw Error(kErrArg, "vector component pointers must be aligned to the element size");
    }
    p.bc_cmb   = bc_cmb;
    p.bc_surf  = bc_surf;
    p.diagonal = diagonal || diag_override;
    p.add      = apply_mode;
    p.tile_y   = tile_y;
    p.chunk_x  = chunk_x;
    p.err      = shell->err_word();
    const int rc = epsdivdiv_apply<T>(p, st);
    if (rc != 0) throw Error(kErrCuda, "epsdivdiv launch failed (" + std::to_string(rc) + ")");
    if (comm_mode == 1) {
        T* comps[3] = {dst[0], dst[1], dst[2]};
        if (interface_sum<T>(L.iface, L.nr(), 3, comps, st) != 0) throw Error(kErrCuda, "interface sum launch failed");
    }
}

template void EpsDivDivOp::apply<double>(const double* const*, double* const*, cudaStream_t, bool) const;
template void EpsDivDivOp::apply<float>(const float* const*, float* const*, cudaStream_t, bool) const;

}  // namespace tn
