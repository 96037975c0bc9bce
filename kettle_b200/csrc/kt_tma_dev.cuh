// kt_tma_dev.cuh — device helpers of the TMA-pipelined block kernels: tensor
// copies between HBM and shared memory (cp.async.bulk.tensor), mbarrier
// completion with bounded waits, bulk-group store completion, named barriers.
// Included by the run-time compiled block kernels (kt_jit.cpp embeds this
// text), so it depends on nothing but the CUDA built-ins.
//
// Every copy here reads or writes this GPU's own memory through a tensor map
// the host encoded over the state; none uses cluster multicast.
#pragma once

#include "kt_complex.cuh"

namespace kt
{

// a CUtensorMap as a kernel parameter (__grid_constant__): 128 bytes, 64-byte aligned
struct alignas(64) KtTmap
{
    unsigned long long w[16];
};

__device__ __forceinline__ uint32_t kt_smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void kt_mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(kt_smem_u32(bar)), "r"(count) : "memory");
}

// the barrier inits visible to the async proxy (the TMA unit) before any copy uses them
__device__ __forceinline__ void kt_fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void kt_mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(kt_smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void kt_mbar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(kt_smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool kt_mbar_try_wait(uint32_t addr, uint32_t parity)
{
    uint32_t ok = 0;
    asm volatile(
        "{\n"
        "    .reg .pred p;\n"
        "    mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "    selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(ok)
        : "r"(addr), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ unsigned long long kt_globaltimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Wait for the phase of `bar` with parity `parity` to complete, for about 2 s
// at most.  On expiry (or at once, when any CTA of the launch has already given
// up) it sets *err and returns false; the caller carries on without the data
// (its results are void and the host reports the error) but keeps to the same
// control flow, so no thread is left waiting at a barrier for one that quit.
__device__ __forceinline__ bool kt_mbar_wait(uint64_t* bar, uint32_t parity, unsigned int* err)
{
    const uint32_t addr = kt_smem_u32(bar);
#pragma unroll 1
    for (int k = 0; k < 32; ++k) {
        if (kt_mbar_try_wait(addr, parity)) {
            return true;
        }
    }
    const unsigned long long t0 = kt_globaltimer();
#pragma unroll 1
    while (true) {
        if (*reinterpret_cast<volatile unsigned int*>(err) != 0u) {
            return false;
        }
        if (kt_mbar_try_wait(addr, parity)) {
            return true;
        }
        if (kt_globaltimer() - t0 > 2000000000ull) {
            atomicOr(err, 1u);
            return false;
        }
    }
}

// consumer writes to a stage buffer made visible to the TMA store that reads it
__device__ __forceinline__ void kt_fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// a barrier over `count` threads (a multiple of 32) with id 1..15; id 0 is __syncthreads
__device__ __forceinline__ void kt_bar_sync(uint32_t id, uint32_t count)
{
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

__device__ __forceinline__ void kt_bulk_commit()
{
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

// the issuing thread's bulk stores have finished reading shared memory
__device__ __forceinline__ void kt_bulk_wait_read0()
{
    asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

// the issuing thread's bulk stores are complete
__device__ __forceinline__ void kt_bulk_wait0()
{
    asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

// Tensor copies of one box: HBM -> shared memory completing on `bar`, and
// shared memory -> HBM in the issuing thread's bulk group.  c[0] is the
// innermost coordinate.
template <int R>
struct KtTma;

template <>
struct KtTma<2>
{
    static __device__ __forceinline__ void load(const KtTmap* tm, void* dst, uint64_t* bar, const int32_t* c)
    {
        asm volatile(
            "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
            "[%4];" ::"r"(kt_smem_u32(dst)),
            "l"(reinterpret_cast<uint64_t>(tm)), "r"(c[0]), "r"(c[1]), "r"(kt_smem_u32(bar))
            : "memory");
    }
    static __device__ __forceinline__ void store(const KtTmap* tm, const void* src, const int32_t* c)
    {
        asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.tile.bulk_group [%0, {%2, %3}], [%1];" ::"l"(
                         reinterpret_cast<uint64_t>(tm)),
                     "r"(kt_smem_u32(src)), "r"(c[0]), "r"(c[1])
                     : "memory");
    }
};

template <>
struct KtTma<3>
{
    static __device__ __forceinline__ void load(const KtTmap* tm, void* dst, uint64_t* bar, const int32_t* c)
    {
        asm volatile(
            "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, "
            "%4}], [%5];" ::"r"(kt_smem_u32(dst)),
            "l"(reinterpret_cast<uint64_t>(tm)), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(kt_smem_u32(bar))
            : "memory");
    }
    static __device__ __forceinline__ void store(const KtTmap* tm, const void* src, const int32_t* c)
    {
        asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%2, %3, %4}], [%1];" ::"l"(
                         reinterpret_cast<uint64_t>(tm)),
                     "r"(kt_smem_u32(src)), "r"(c[0]), "r"(c[1]), "r"(c[2])
                     : "memory");
    }
};

template <>
struct KtTma<4>
{
    static __device__ __forceinline__ void load(const KtTmap* tm, void* dst, uint64_t* bar, const int32_t* c)
    {
        asm volatile(
            "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, "
            "%4, %5}], [%6];" ::"r"(kt_smem_u32(dst)),
            "l"(reinterpret_cast<uint64_t>(tm)), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(kt_smem_u32(bar))
            : "memory");
    }
    static __device__ __forceinline__ void store(const KtTmap* tm, const void* src, const int32_t* c)
    {
        asm volatile(
            "cp.async.bulk.tensor.4d.global.shared::cta.tile.bulk_group [%0, {%2, %3, %4, %5}], [%1];" ::"l"(
                reinterpret_cast<uint64_t>(tm)),
            "r"(kt_smem_u32(src)), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3])
            : "memory");
    }
};

template <>
struct KtTma<5>
{
    static __device__ __forceinline__ void load(const KtTmap* tm, void* dst, uint64_t* bar, const int32_t* c)
    {
        asm volatile(
            "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, "
            "%4, %5, %6}], [%7];" ::"r"(kt_smem_u32(dst)),
            "l"(reinterpret_cast<uint64_t>(tm)), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(c[4]),
            "r"(kt_smem_u32(bar))
            : "memory");
    }
    static __device__ __forceinline__ void store(const KtTmap* tm, const void* src, const int32_t* c)
    {
        asm volatile(
            "cp.async.bulk.tensor.5d.global.shared::cta.tile.bulk_group [%0, {%2, %3, %4, %5, %6}], [%1];" ::"l"(
                reinterpret_cast<uint64_t>(tm)),
            "r"(kt_smem_u32(src)), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(c[4])
            : "memory");
    }
};

}  // namespace kt
