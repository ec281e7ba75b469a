// Row pipeline of the stencil kernels: every CTA owns a strip of W columns
// and a range of rows; for each row it needs, warp 0 issues 1-D bulk copies
// (cp.async.bulk global -> shared, completion counted on an mbarrier) into a
// ring of Q shared-memory slots, Q-1 rows ahead of the row being computed.
// No cluster multicast is used anywhere.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace dn {

// Bounded wait: ~1 s of try_wait polling before the kernel gives up with an error flag.
#define DN_SPIN_LIMIT (1 << 22)

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// dst (shared) and src (global) 16-byte aligned, bytes a multiple of 16
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// waits for the phase `parity` of `bar`; returns false when the spin limit ran out
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity)
{
    for (int k = 0; k < DN_SPIN_LIMIT; k++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// One copy of an item: a row segment of one field.
struct RowCopy {
    const float *src;
    unsigned dst;      // float offset inside the slot
    unsigned bytes;
};

// Shared state of a CTA's pipeline.
template <int Q>
struct Pipe {
    uint64_t *bars;
    float *slots;
    int slot_floats;

    __device__ __forceinline__ void init(float *smem, int slot_floats_)
    {
        slot_floats = slot_floats_;
        slots = smem;
        bars = (uint64_t *)(smem + (size_t)Q * slot_floats_);
        if (threadIdx.x == 0) {
            for (int q = 0; q < Q; q++) mbar_init(&bars[q], 1);
            mbar_fence_init();
        }
        __syncthreads();
    }
    __device__ __forceinline__ float *slot(int item) const { return slots + (size_t)(item % Q) * slot_floats; }

    // warp 0 only: lane 0 arms the slot's barrier with the item's byte count,
    // lanes 0..n-1 each issue one copy
    __device__ __forceinline__ void issue(int item, const RowCopy &mine, int n, unsigned total_bytes)
    {
        const int lane = threadIdx.x & 31;
        uint64_t *bar = &bars[item % Q];
        if (lane == 0) mbar_arrive_expect_tx(bar, total_bytes);
        __syncwarp();
        if (lane < n) bulk_g2s(slot(item) + mine.dst, mine.src, mine.bytes, bar);
    }

    // all threads: bounded wait for `item`; returns false (uniformly) on time-out
    __device__ __forceinline__ bool wait(int item)
    {
        const bool ok = mbar_wait_bounded(&bars[item % Q], (unsigned)((item / Q) & 1));
        return !__syncthreads_or(!ok);
    }

    // error exit: drain the items still in flight (bounded) so no copy lands after the CTA exits
    __device__ __forceinline__ void drain(int first, int last)
    {
        for (int it = first; it <= last; it++) mbar_wait_bounded(&bars[it % Q], (unsigned)((it / Q) & 1));
        __syncthreads();
    }
};

}   // namespace dn
