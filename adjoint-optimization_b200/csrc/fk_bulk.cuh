// fk_bulk.cuh -- tile windows into shared memory through the bulk-copy (TMA)
// engine, for sm_100a.
//
// A window is rows x WIDTH doubles of each of the three field planes (row
// pitch ld, plane pitch `plane` in global memory; row pitch WIDTH, plane pitch
// RCAP * WIDTH in shared memory).  Every row is one cp.async.bulk, completing
// on an mbarrier in shared memory.  A row must start on a 16-byte boundary and
// be a multiple of 16 bytes long: the callers check the addresses and fall back
// to vector loads otherwise.
//
// Protocol (all threads of the CTA):
//   bar = bulk_begin(&smem_u64);  __syncthreads();
//   bulk_arrive(bar, bytes);      __syncthreads();   // thread 0 posts the count
//   bulk_issue<...>(bar, ...);    // one or more windows, bytes in total
//   ok = bulk_wait(bar);          // false: the bounded wait expired
// or, for one outcome across the CTA (and the fault word set on expiry),
//   ok = bulk_wait_cta(bar, fault);
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace fkadj {

// Shared-memory address of the CTA's mbarrier, initialised by thread 0 for one
// arrival; the caller synchronises the CTA before its first use.
__device__ __forceinline__ uint32_t bulk_begin(uint64_t* bar) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(bar);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(a) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    return a;
}

// Bytes of a rows x WIDTH window of the three planes.
template <int WIDTH>
__device__ __forceinline__ uint32_t bulk_bytes(int rows) {
    static_assert((WIDTH * 8) % 16 == 0, "bulk rows must be 16-byte multiples");
    return 3u * (uint32_t)rows * WIDTH * 8u;
}

// Thread 0 arrives on the barrier with the transfer's byte count; the CTA
// synchronises before the copies are issued.
__device__ __forceinline__ void bulk_arrive(uint32_t bar, uint32_t bytes) {
    if (threadIdx.x == 0)
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// Issues the copies of one window, spread over the NT threads.
template <int RCAP, int WIDTH, int NT>
__device__ __forceinline__ void bulk_issue(uint32_t bar, double* dst, const double* src, int ld, long long plane,
                                           int rows) {
    constexpr int RN = RCAP * WIDTH;
    for (int t = threadIdx.x; t < 3 * rows; t += NT) {
        const int f = t / rows, r = t - f * rows;
        const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst + f * RN + r * WIDTH);
        const size_t gsrc = __cvta_generic_to_global(src + f * plane + (long long)r * ld);
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(d),
            "l"(gsrc), "n"(WIDTH * 8), "r"(bar)
            : "memory");
    }
}

__device__ __forceinline__ uint64_t bulk_now_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Waits for the phase of the barrier with the given parity (0 for its first
// transfer, then 1, 0, ... when one barrier serves a sequence of transfers)
// for at most about limit_ns of wall time (and at most 2^22 polls); returns
// false when the wait expired.  Then the posted bytes did not all arrive in
// time: the tile is incomplete, the caller records the error and the host
// discards the call's results.
__device__ __forceinline__ bool bulk_wait(uint32_t bar, uint64_t limit_ns = 1000000000ull, uint32_t parity = 0) {
    const uint64_t t0 = bulk_now_ns();
    for (int it = 0; it < (1 << 22); ++it) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
        if (bulk_now_ns() - t0 > limit_ns) break;
    }
    return false;
}

// bulk_wait for all threads of a CTA, with one outcome for all of them: true
// when the posted bytes arrived.  When the wait expired in any thread, thread
// 0 sets *fault (when non-null), the CTA waits once more, again bounded, for
// copies still in flight, and every thread gets false: the window is
// incomplete and the caller returns without computing or storing anything.
// Copies that land after the second wait expired would write into shared
// memory the CTA no longer owns; that is the risk this path leaves open.
__device__ __forceinline__ bool bulk_wait_cta(uint32_t bar, unsigned* fault, uint64_t limit_ns = 1000000000ull,
                                              uint32_t parity = 0) {
    const bool ok = bulk_wait(bar, limit_ns, parity);
    if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0 && fault) atomicOr(fault, 1u);
        bulk_wait(bar, limit_ns, parity);
        return false;
    }
    return true;
}

}  // namespace fkadj
