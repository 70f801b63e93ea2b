// Grid-wide barrier for persistent cooperative kernels.
//
// One monotone arrival counter (zero at launch): every block adds 1 per
// barrier and waits until the counter reaches (barriers so far) x (blocks).
// No block resets anything, so there is one atomic per block and barrier and
// the waiters poll a single word.  The wait gives up after a limit (two seconds
// by default), or as soon as another block has set the device error word, and then reports
// failure so that the kernel can return instead of hanging.
#pragma once
#include "kcommon.cuh"

namespace igr {

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// `epoch` is a per-thread register starting at 0, advanced identically by
// every thread of the block.  Returns false on timeout or a reported error.
// `limit_ns` bounds the wait; `phantom` (a test hook, normally 0) adds
// arrivals that never come, so that the wait runs out by construction.
__device__ __forceinline__ bool grid_sync(unsigned *count, int *err, unsigned &epoch,
                                          unsigned long long limit_ns = 2000000000ull, unsigned phantom = 0) {
    __shared__ int s_ok;
    __syncthreads();
    epoch += gridDim.x + phantom;
    if (threadIdx.x == 0) {
        int ok = 1;
        __threadfence();
        unsigned v = atomicAdd(count, 1u) + 1u;
        const unsigned long long t0 = global_ns();
        while ((int)(v - epoch) < 0) {
            asm volatile("ld.acquire.gpu.u32 %0, [%1];" : "=r"(v) : "l"(count) : "memory");
            if ((int)(v - epoch) >= 0) break;
            if (*(volatile int *)err) { ok = 0; break; }
            if (global_ns() - t0 > limit_ns) {
                set_error(err, ERR_TIMEOUT);
                ok = 0;
                break;
            }
        }
        __threadfence();
        if (ok && *(volatile int *)err) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

}  // namespace igr
