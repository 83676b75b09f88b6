// Bounded grid-wide barrier for cooperative launches (all CTAs co-resident).
#pragma once

#include <cuda/atomic>
#include <cuda_runtime.h>

#include "xpbd_common.cuh"

namespace xpbd {

constexpr unsigned kSpinLimit = 1u << 21;  // polls of ~0.5 us (L2 round trip + 32 ns sleep): about a second

// Grid-wide barrier over gridDim.x co-resident CTAs (count, generation in
// sync[0..1]).  __syncthreads orders the CTA's writes before thread 0's
// acquire-release arrival; the release of the new generation and the
// acquiring polls carry them to the other CTAs, whose __syncthreads passes
// them on to their threads.  Bounded: after kSpinLimit polls it sets the
// timeout bit, and once that bit is set no CTA waits again.
__device__ __forceinline__ void grid_barrier(uint32_t* sync, int32_t* status) {
    __syncthreads();
    if (threadIdx.x == 0) {
        cuda::atomic_ref<uint32_t, cuda::thread_scope_device> cnt(sync[0]), gen(sync[1]);
        cuda::atomic_ref<int32_t, cuda::thread_scope_device> st(*status);
        if ((st.load(cuda::memory_order_relaxed) & XPBD_STATUS_BARRIER_TIMEOUT) == 0) {
            const uint32_t g = gen.load(cuda::memory_order_relaxed);
            if (cnt.fetch_add(1u, cuda::memory_order_acq_rel) == gridDim.x - 1) {
                cnt.store(0u, cuda::memory_order_relaxed);
                gen.fetch_add(1u, cuda::memory_order_release);
            } else {
                uint32_t spins = 0;
                while (gen.load(cuda::memory_order_acquire) == g) {
                    if (++spins > kSpinLimit) {
                        st.fetch_or(XPBD_STATUS_BARRIER_TIMEOUT, cuda::memory_order_relaxed);
                        break;
                    }
                    __nanosleep(32);
                }
            }
        }
    }
    __syncthreads();
}

}  // namespace xpbd
