// Device-side helpers shared by the gridder's kernels (sm_100a).
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace b200 {

// Bits OR-ed into the workspace's device status word by kernel self-checks.
enum : unsigned
{
    DEV_ERR_GRID_INDEX = 1u << 0,   // a flush would have left the grid
    DEV_ERR_SLAB_INDEX = 1u << 1,   // a kernel tap would have left its slab
    DEV_ERR_TIMEOUT = 1u << 2,      // a bounded mbarrier wait expired
    DEV_ERR_TASK = 1u << 3          // malformed task bounds
};

// Iteration limit of every device-side spin-wait.  mbarrier.try_wait
// suspends for a hardware-defined interval per attempt, so this bounds a
// wait at well under a minute even in the worst case.
constexpr unsigned kSpinLimit = 1u << 22;

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// ---------------------------------------------------------------------------
// Grid atomics: fire-and-forget reductions (no return value).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void red_add_c(float* addr, float re, float im)
{
    // One 8-byte vector reduction per complex cell (sm_90+).
    asm volatile("red.relaxed.gpu.global.add.v2.f32 [%0], {%1, %2};"
                 :: "l"(addr), "f"(re), "f"(im) : "memory");
}

__device__ __forceinline__ void red_add_c(double* addr, double re, double im)
{
    asm volatile("red.relaxed.gpu.global.add.f64 [%0], %1;"
                 :: "l"(addr), "d"(re) : "memory");
    asm volatile("red.relaxed.gpu.global.add.f64 [%0], %1;"
                 :: "l"(addr + 1), "d"(im) : "memory");
}

// ---------------------------------------------------------------------------
// mbarrier and bulk (non-tensor) TMA copies into this CTA's shared memory.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;"
                 :: "r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar,
                                                      uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                 :: "r"(smem_addr(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done) : "r"(smem_addr(bar)), "r"(parity) : "memory");
    return done != 0;
}

// Bounded wait; returns false when the iteration limit ran out.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar,
                                                  uint32_t parity,
                                                  unsigned limit = kSpinLimit)
{
    for (unsigned i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// Orders this thread's earlier generic-proxy shared-memory accesses (made
// visible to it by a preceding __syncthreads) before later async-proxy
// writes into the same shared memory.
__device__ __forceinline__ void fence_proxy_async_shared()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Global -> shared bulk copy completing on `bar`.  dst, src and bytes must
// be multiples of 16.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src,
                                              uint32_t bytes, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
        "[%0], [%1], %2, [%3];"
        :: "r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// ---------------------------------------------------------------------------
// Kernel-value storage types and their widening loads.
// ---------------------------------------------------------------------------
template <typename KT> struct KernelLoad;

template <> struct KernelLoad<float2>
{
    using Wide = float2;
    __device__ __forceinline__ static float2 get(const float2& k) { return k; }
};
template <> struct KernelLoad<double2>
{
    using Wide = double2;
    __device__ __forceinline__ static double2 get(const double2& k) { return k; }
};
template <> struct KernelLoad<__half2>
{
    using Wide = float2;
    __device__ __forceinline__ static float2 get(const __half2& k)
    {
        return __half22float2(k);
    }
};
template <> struct KernelLoad<__nv_bfloat162>
{
    using Wide = float2;
    __device__ __forceinline__ static float2 get(const __nv_bfloat162& k)
    {
        return __bfloat1622float2(k);
    }
};

// ---------------------------------------------------------------------------
// Warp and block reductions.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace b200
