// Divergence B in Replace + CommunicateAdditively mode with its per-wedge
// scratch in a fixed, statically allocated device array instead of a buffer
// allocated on first use.
//
// Some callers cannot allocate device memory at the time they apply the
// operator: code running while a memory budget is frozen (a pool that has
// been carved up front and must not grow), a real-time loop in which an
// allocation's implicit device synchronisation would stall other streams, or
// a host thread that must not take the driver's allocation locks. For them
// this entry point uses only a file-scope scratch array whose device address
// is looked up once per device.
//
// Limits and rules:
//   * the scratch holds kScratchBytes = 8 MiB, i.e. 2 values per fine cell:
//     velocity levels up to 5 in FP64 (327,680 cells -> 5 MiB) and up to 5 in
//     FP32; larger levels are rejected with TN_ERR_ARG;
//   * nothing in the scratch needs to start at zero: the first kernel writes
//     every value the second one reads; the output is zeroed by the call;
//   * the scratch is shared by all calls on a device, so calls that overlap
//     in time (different streams, no ordering between them) race on it; order
//     them on one stream or synchronise between them;
//   * the first call on a device does the set-up: it looks up the scratch
//     address (a driver query; with lazy module loading the driver may load
//     this module and its static array at that point); make that first call
//     before any stream capture.
#include <mutex>

#include "../../include/terra_b200.h"
#include "tn_kernels.hpp"
#include "tn_runtime.hpp"

namespace tn {
Shell* shell_of(tn_shell* s);
void   set_last_error(const std::string& message);

namespace {

constexpr size_t kScratchBytes = size_t(8) << 20;
constexpr int    kMaxDevices   = 64;

static __device__ __align__(256) unsigned char g_wedge_scratch[kScratchBytes];

// device address of g_wedge_scratch per device ordinal, looked up once
void* scratch_address(int device)
{
    static std::mutex mu;
    static void*      addr[kMaxDevices] = {};
    std::lock_guard<std::mutex> lock(mu);
    if (device < 0 || device >= kMaxDevices) throw Error(kErrArg, "device ordinal out of range");
    if (addr[device] == nullptr) {
        void*             p  = nullptr;
        const cudaError_t rc = cudaGetSymbolAddress(&p, g_wedge_scratch);
        if (rc != cudaSuccess || p == nullptr) {
            cudaGetLastError();
            throw Error(kErrCuda, std::string("cudaGetSymbolAddress of the static scratch failed: ") +
                                      cudaGetErrorString(rc));
        }
        addr[device] = p;
    }
    return addr[device];
}

template <typename T>
void apply(const DeviceLevel& L, const DeviceLevel& Lc, int bc_cmb, int bc_surf, const T* const* u, T* p,
           cudaStream_t st)
{
    int device = 0;
    cuda_check(cudaGetDevice(&device), "current device");
    T* scratch = static_cast<T*>(scratch_address(device));
    cuda_check(cudaMemsetAsync(p, 0, sizeof(T) * static_cast<size_t>(Lc.nodes()), st), "zero output");
    CouplingLaunch<T> c;
    c.nl      = L.nl();
    c.nr      = L.nr();
    c.coords  = L.coords<T>();
    c.colgeo  = L.colgeo<T>();
    c.radgeo  = L.radgeo<T>();
    c.radii   = L.radii<T>();
    c.bc_cmb  = bc_cmb;
    c.bc_surf = bc_surf;
    for (int k = 0; k < 3; ++k) c.u[k] = u[k];
    c.p_out         = p;
    c.wedge_scratch = scratch;
    if (divergence_apply<T>(c, st) != 0) throw Error(kErrCuda, "divergence launch failed");
    T* pc[1] = {p};
    if (interface_sum<T>(Lc.iface, Lc.nr(), 1, pc, st) != 0) throw Error(kErrCuda, "interface sum launch failed");
}

}  // namespace
}  // namespace tn

extern "C" int tn_divergence_apply_noalloc(tn_shell* shell, int velocity_level, int precision, int bc_cmb,
                                           int bc_surface, const void* const* u_dev, void* p_dev, void* stream)
{
    try {
        tn::set_last_error("");
        tn::Shell* sh = tn::shell_of(shell);
        if (!sh || !u_dev || !p_dev) throw tn::Error(tn::kErrArg, "NULL argument");
        if (bc_cmb < 0 || bc_cmb > 2 || bc_surface < 0 || bc_surface > 2)
            throw tn::Error(tn::kErrArg, "invalid boundary condition");
        if (precision != TN_F64 && precision != TN_F32)
            throw tn::Error(tn::kErrArg, "precision must be TN_F64 or TN_F32");
        if (velocity_level < 1) throw tn::Error(tn::kErrArg, "the velocity level needs a coarser pressure level");
        const tn::DeviceLevel& L  = sh->level(velocity_level);
        const tn::DeviceLevel& Lc = sh->level(velocity_level - 1);
        const size_t           es = precision == TN_F64 ? sizeof(double) : sizeof(float);
        const size_t           need = 2 * es * static_cast<size_t>(L.cells());
        if (need > tn::kScratchBytes)
            throw tn::Error(tn::kErrArg, "level needs " + std::to_string(need) + " bytes of scratch; the static scratch "
                                         "holds " + std::to_string(tn::kScratchBytes) +
                                         " bytes (velocity levels up to 5)");
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        if (precision == TN_F64)
            tn::apply<double>(L, Lc, bc_cmb, bc_surface, reinterpret_cast<const double* const*>(u_dev),
                              static_cast<double*>(p_dev), st);
        else
            tn::apply<float>(L, Lc, bc_cmb, bc_surface, reinterpret_cast<const float* const*>(u_dev),
                             static_cast<float*>(p_dev), st);
        return TN_OK;
    } catch (const tn::Error& e) {
        tn::set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        tn::set_last_error(e.what());
        return TN_ERR_ARG;
    }
}
