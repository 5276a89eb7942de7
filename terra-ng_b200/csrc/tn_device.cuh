// Shared device helpers for the sm_100a kernels: layout arithmetic, TMA bulk
// copies with bounded mbarrier waits, and the error flag every bounded wait
// reports to.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace tn {


// Device-side error codes written to the per-context error word.
enum DeviceError : int {
    kDevOk             = 0,
    kDevMbarrierTimeout = 1,
    kDevBadLaunch      = 2,
};

// Nodal index (diamond, x, y, r), r fastest (grid/grid_types.hpp:12-30).
__host__ __device__ __forceinline__ int64_t node_index(int nl, int nr, int d, int x, int y, int r)
{
    return ((static_cast<int64_t>(d) * nl + x) * nl + y) * nr + r;
}

// ---------------------------------------------------------------------------
// mbarrier + bulk copy (cp.async.bulk, no multicast).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_barrier_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity), "r"(100000u)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t global_timer_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Wait for phase `parity` of `bar`, giving up after ~`limit_ns`. Returns false
// on timeout; the caller records the error and stops using the buffer.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint64_t limit_ns = 1000000000ull)
{
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_timer_ns();
    while (true) {
        if (mbar_try_wait(bar, parity)) return true;
        if (global_timer_ns() - t0 > limit_ns) return false;
    }
}

// 1-D bulk copy global -> this CTA's shared memory, completing on `bar`.
// dst and src must be 16-byte aligned and bytes a multiple of 16.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ void report_error(int* err, int code)
{
    if (err) atomicCAS(err, 0, code);
}

template <typename T>
__device__ __forceinline__ T shfl_up(T v, int delta)
{
    return __shfl_up_sync(0xffffffffu, v, delta);
}
template <typename T>
__device__ __forceinline__ T shfl_down(T v, int delta)
{
    return __shfl_down_sync(0xffffffffu, v, delta);
}

}  // namespace tn
