// k_gridbar.cuh -- a grid-wide barrier for cooperative launches (every CTA
// co-resident), used by the resident SOR kernel.  Every wait is bounded: a barrier that gives up sets a shared
// error flag, so that the other CTAs leave at their next wait.
#pragma once

#include "ntcfd_common.cuh"

namespace ntcfd {

struct GridBar {
    // low 32 bits: arrivals since the launch began; high 32 bits: the sum over the
    // sweeps' closing barriers of the CTAs whose max |change| was above zeta, plus
    // 2^20 per CTA whose max was not finite (k_defect zeroes the word)
    unsigned long long word;
    int err;
    int pad;
};

constexpr unsigned int kBarrierPolls = 20000000u;   // ~1-2 s of polling without sleep

__device__ __forceinline__ unsigned long long ld_acquire(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void red_add_release(unsigned long long* p, unsigned long long v) {
    asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ int vload(const int* p) { return *(const volatile int*)p; }

// Grid-wide barrier of one cooperative launch, split into arrive and wait so
// that a CTA can work between the two.  One 64-bit word counts the arrivals of
// the launch in its low half: each CTA adds 1 per barrier with a release
// reduction (after a CTA barrier, so the CTA's earlier global writes are
// published) and does not wait for the add to come back; the n-th barrier of
// the launch is passed once the low half reaches n * nblocks.  A CTA may add
// flags to the high half with its arrival (flags << 32); they are summed over
// the launch, and a waiter reads the sum as it sees the barrier pass.  Waiting
// polls the word with acquire loads, checks the shared error flag every 1024
// polls and gives up after kBarrierPolls polls, setting the flag so that every
// CTA leaves at its next wait.  Returns false on failure.
__device__ __forceinline__ void grid_arrive(GridBar* b, unsigned int& nbar, unsigned int flags = 0u) {
    __syncthreads();
    if (threadIdx.x == 0) red_add_release(&b->word, 1ull | ((unsigned long long)flags << 32));
    ++nbar;
}

// With hi non-null, thread 0 also stores the high half of the word as it saw
// the barrier pass to *hi before the closing CTA barrier, so every thread sees it.
__device__ __forceinline__ bool grid_wait(GridBar* b, unsigned int nbar, unsigned int nblocks, int* s_flag,
                                          unsigned int* hi = nullptr) {
    if (threadIdx.x == 0) {
        const unsigned int target = nbar * nblocks;
        int fail = 0;
        unsigned int polls = 0;
        unsigned long long w;
        while ((int)((unsigned int)(w = ld_acquire(&b->word)) - target) < 0) {
            if ((++polls & 1023u) == 0u) {
                if (vload(&b->err) != 0) { fail = 1; break; }
                if (polls > kBarrierPolls) {
                    atomicExch(&b->err, 1);
                    fail = 1;
                    break;
                }
            }
        }
        *s_flag = fail;
        if (hi) *hi = (unsigned int)(w >> 32);
    }
    __syncthreads();
    return *s_flag == 0;
}

__device__ __forceinline__ bool grid_sync(GridBar* b, unsigned int& nbar, unsigned int nblocks, int* s_flag,
                                          unsigned int flags = 0u, unsigned int* hi = nullptr) {
    grid_arrive(b, nbar, flags);
    return grid_wait(b, nbar, nblocks, s_flag, hi);
}

}  // namespace ntcfd
