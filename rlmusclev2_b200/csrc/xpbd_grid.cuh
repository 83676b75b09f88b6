// Bounded grid-wide barrier for cooperative launches (all CTAs co-resident).
#pragma once

#include <cuda_runtime.h>

#include "xpbd_common.cuh"

namespace xpbd {

constexpr unsigned kSpinLimit = 1u << 21;  // polls of ~0.5 us (one L2 round trip each): about a second
constexpr unsigned kSpinCheck = 64u;       // polls between two reads of the status word

// Barrier words (four uint32, zero before the first launch that uses them):
//   [0], [1]  arrival counters; consecutive launches alternate between them
//   [2]       free for the kernel (the persistent pass keeps its ring phase there)
//   [3]       which counter the next launch uses (bit 0)
// A launch reads [3] once per CTA before its first arrival, counts every
// arrival into its counter and waits until the counter reaches k * gridDim.x
// at its k-th barrier; the counter only grows within a launch, so the last
// arrival itself releases the barrier (no reset, no second word on the
// critical path).  Block 0 zeroes the other counter at the start (the
// previous launch, which used it, has finished; the next one has not begun)
// and flips [3] after its last barrier, when every CTA has read it.
struct GridBarrier {
    uint32_t* cnt;
    uint32_t target;
    uint32_t par;
};

__device__ __forceinline__ GridBarrier grid_barrier_begin(uint32_t* sync) {
    GridBarrier b;
    b.par = __ldcg(sync + 3) & 1u;
    b.cnt = sync + b.par;
    b.target = 0u;
    if (blockIdx.x == 0 && threadIdx.x == 0) sync[b.par ^ 1u] = 0u;
    return b;
}

// Called after the launch's last barrier (a launch takes at least one).
__device__ __forceinline__ void grid_barrier_end(uint32_t* sync, const GridBarrier& b) {
    if (blockIdx.x == 0 && threadIdx.x == 0) sync[3] = b.par ^ 1u;
}

__device__ __forceinline__ void red_release_add(uint32_t* p, uint32_t v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// __syncthreads orders the CTA's writes before thread 0's release arrival;
// the acquiring polls that see the full count carry every CTA's writes to
// this CTA, whose second __syncthreads passes them on to its threads.
// Bounded: after kSpinLimit polls the CTA sets XPBD_STATUS_BARRIER_TIMEOUT
// and stops waiting; a CTA that finds the bit set while it waits stops too,
// so after a timeout every later barrier of the launch ends within
// kSpinCheck polls.
__device__ __forceinline__ void grid_barrier(GridBarrier& b, int32_t* status) {
    __syncthreads();
    if (threadIdx.x == 0) {
        b.target += gridDim.x;
        red_release_add(b.cnt, 1u);
        uint32_t spins = 0;
        while (ld_acquire(b.cnt) < b.target) {
            if (++spins % kSpinCheck == 0u) {
                if (spins > kSpinLimit) {
                    atomicOr(status, XPBD_STATUS_BARRIER_TIMEOUT);
                    break;
                }
                if (*reinterpret_cast<volatile int32_t*>(status) & XPBD_STATUS_BARRIER_TIMEOUT) break;
                __nanosleep(32);
            }
        }
    }
    __syncthreads();
}

// Neighbour synchronisation of the persistent pass: tile `self` publishes
// that it finished iteration `it` (its counter becomes c0 + it + 1, c0 being
// the counter at launch start, equal for all tiles) and waits until each of
// its neighbours has published at least that.  A tile only reads ring slots
// of vertices it shares with those neighbours, so this orders every partial
// sum it reads (and, two iterations on, every clear) as the grid-wide barrier
// does, without waiting for tiles elsewhere.  The lanes of warp 0 poll the
// neighbour counters in parallel.  Bounded like grid_barrier: after kSpinLimit
// polls the bit is set and the wait ends; a set bit ends later waits early.
__device__ __forceinline__ void st_release(uint32_t* p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ void neighbour_sync(uint32_t* cnt, const int32_t* nbr, int n_nbr, int self, uint32_t target,
                                               int32_t* status) {
    __syncthreads();
    if (threadIdx.x < 32) {
        if (threadIdx.x == 0) st_release(cnt + self, target);
        for (int j = int(threadIdx.x); j < n_nbr; j += 32) {
            const uint32_t* c = cnt + nbr[j];
            uint32_t spins = 0;
            while (int32_t(ld_acquire(c) - target) < 0) {
                if (++spins % kSpinCheck == 0u) {
                    if (spins > kSpinLimit) {
                        atomicOr(status, XPBD_STATUS_BARRIER_TIMEOUT);
                        break;
                    }
                    if (*reinterpret_cast<volatile int32_t*>(status) & XPBD_STATUS_BARRIER_TIMEOUT) break;
                    __nanosleep(32);
                }
            }
        }
        __syncwarp();
    }
    __syncthreads();
}

}  // namespace xpbd
