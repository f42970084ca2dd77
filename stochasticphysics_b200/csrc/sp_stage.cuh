// sp_stage.cuh — injected Wiener increments streamed from HBM into shared memory.
//
// In injection mode every particle-step reads Mn increments from dW[S][Mn][Np] (HBM,
// far larger than L2).  Each warp stages the rows of its own 32 particles a few steps
// ahead: one lane per row issues a bulk asynchronous copy (cp.async.bulk, global ->
// shared, completion counted in bytes on an mbarrier) of 32 consecutive increments,
// kStep steps per stage and kStages stages in a ring, so about (kStages - 1) kStep Mn
// rows per warp are in flight while the warp computes, without holding any of them in
// registers.  The ring is sized so that four 128-thread CTAs fit an SM (FP64, noise
// dimension 3: 9 KB per warp).  The copies read this GPU's own memory only and use no
// multicast.
//
// Every wait on a stage is bounded by a clock budget.  A stage that does not arrive in
// time sets EnsCtl::fault, the warp waits (bounded again) for the copies it still has in
// flight, and the kernel's caller sees SP_ERR_DEVICE_TIMEOUT when it reads the ensemble.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "sp_types.h"

namespace sp {

constexpr long long kStageWaitCycles = 4000000000ll;  // about 2 s at the B200's clock

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    return done != 0;
}
// waits for phase `parity` of the barrier for at most kStageWaitCycles
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity) {
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > kStageWaitCycles) return false;
    return true;
}
// one row of `bytes` from global to shared memory, completing on the barrier
__device__ __forceinline__ void bulk_copy_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(dst), "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

// The increments of one warp's 32 particles for the steps of one tile, in order.
template <class R, int Mn>
struct DwStream {
    static constexpr int kStep = 4;    // steps per stage
    static constexpr int kStages = 3;  // stages in the ring
    static constexpr int kRow = 32 * static_cast<int>(sizeof(R));
    static constexpr int kStageBytes = kStep * Mn * kRow;
    static_assert(kRow % 16 == 0, "bulk copies move multiples of 16 bytes");
    static_assert(kStep * Mn <= 32, "one lane issues each row of a stage");

    // dynamic shared memory of a CTA of `threads` threads
    static constexpr size_t smem_bytes(int threads) { return static_cast<size_t>(threads / 32) * kStages * kStageBytes; }

    R* buf;               // this warp's ring: [kStages][kStep][Mn][32]
    uint32_t bar0;        // its first barrier (8 bytes apart)
    unsigned int q_issue, q_done;  // stages issued / consumed by this warp (ring slot = q % kStages)
    const R* src;         // increments of the tile's first step for the warp's particles
    unsigned long long Np, nsteps, pos;
    bool ok;

    // lane 0 initialises the warp's barriers once per kernel
    __device__ __forceinline__ void init(R* warp_buf, uint64_t* warp_bars) {
        buf = warp_buf;
        bar0 = smem_addr(warp_bars);
        q_issue = q_done = 0;
        ok = true;
        if ((threadIdx.x & 31) == 0) {
#pragma unroll
            for (int s = 0; s < kStages; ++s) mbar_init(bar0 + 8 * s, 1);
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        __syncwarp();
    }

    // stage k of the tile (steps k kStep ...) into ring slot q_issue % kStages
    __device__ __forceinline__ void issue(unsigned long long k) {
        const int slot = static_cast<int>(q_issue % kStages);
        const unsigned long long j0 = k * kStep;
        const int steps = static_cast<int>(min(static_cast<unsigned long long>(kStep), nsteps - j0));
        const int rows = steps * Mn;
        const uint32_t bar = bar0 + 8 * slot;
        const int lane = threadIdx.x & 31;
        if (lane == 0) mbar_expect_tx(bar, static_cast<uint32_t>(rows * kRow));
        __syncwarp();
        if (lane < rows) {
            // the generic-proxy reads of this slot's previous stage precede the new copy
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            const int st = lane / Mn, m = lane % Mn;
            const R* g = src + ((j0 + st) * Mn + m) * Np;
            bulk_copy_g2s(smem_addr(buf + (slot * kStep + st) * Mn * 32 + m * 32), g, kRow, bar);
        }
        ++q_issue;
    }

    // a new tile: the warp's particles start at `first`, increments of steps s0 ...
    __device__ __forceinline__ void begin(const R* dw, unsigned long long np, unsigned long long first,
                                          unsigned long long s0, unsigned long long n) {
        Np = np;
        nsteps = n;
        pos = 0;
        src = dw + s0 * Mn * np + first;
        const unsigned long long stages = (n + kStep - 1) / kStep;
        for (unsigned long long k = 0; k < stages && k < kStages; ++k) issue(k);
    }

    // waits, bounded, for every stage still in flight (after a timeout)
    __device__ void drain() {
        while (q_done < q_issue) {
            const int slot = static_cast<int>(q_done % kStages);
            mbar_wait_bounded(bar0 + 8 * slot, (q_done / kStages) & 1u);
            ++q_done;
        }
    }

    // the increments of the next step for this lane's particle; false once a stage has
    // timed out (uniform across the warp)
    __device__ __forceinline__ bool next(R* w) {
        const int within = static_cast<int>(pos % kStep);
        const int slot = static_cast<int>(q_done % kStages);
        if (within == 0) {
            const bool mine = mbar_wait_bounded(bar0 + 8 * slot, (q_done / kStages) & 1u);
            if (!__all_sync(0xffffffffu, mine)) {
                ok = false;
                return false;
            }
        }
        const R* row = buf + (slot * kStep + within) * Mn * 32 + (threadIdx.x & 31);
#pragma unroll
        for (int m = 0; m < Mn; ++m) w[m] = row[m * 32];
        ++pos;
        if (within == kStep - 1 || pos == nsteps) {  // the stage is consumed: refill its slot
            __syncwarp();
            ++q_done;
            const unsigned long long k = (pos + kStep - 1) / kStep - 1 + kStages;  // stage index in the tile
            if (k * kStep < nsteps) issue(k);
        }
        return true;
    }
};

}  // namespace sp
