// Tensor-core GEMM and the small kernels of the learned coarse correction
// (per-cage-vertex MLP: forward, backward and Adam, BF16 operands, FP32
// accumulation).
//
// xpbd_gemm_bf16: C[m][n] = sum_k A[m][k] * B[n][k] on the 5th-generation
// tensor cores (tcgen05.mma kind::f16, cta_group::1, accumulator in tensor
// memory), one CTA per 128-row x n_tile block of C:
//   * A and B are row-major along k (K-major), k a multiple of 64.  Each
//     64-wide k block of A (128 x 64) and B (n_tile x 64) is copied from global
//     memory into shared memory in the canonical no-swizzle K-major layout
//     (8-row x 16-byte core matrices; leading byte offset 128 B between the two
//     k halves of an MMA, stride byte offset 1024 B between 8-row groups);
//   * two shared-memory stages: while the tensor core works on stage s (four
//     128 x n_tile x 16 MMAs issued by one thread, completion tracked by an
//     mbarrier through tcgen05.commit), the CTA loads stage s+1;
//   * the epilogue reads the accumulator with tcgen05.ld (warp w owns TMEM
//     lanes 32w..32w+31 = rows of the tile) and applies bias, the GELU
//     derivative of a stored pre-activation (backward), GELU, and writes FP32
//     and/or BF16 (row-major and/or transposed) outputs.
// Every mbarrier wait is bounded; on timeout the status word gets
// XPBD_STATUS_MMA_TIMEOUT, the CTA waits (bounded) once more for its MMAs and
// frees its tensor memory before returning.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "xpbd_common.cuh"

using namespace xpbd;

namespace {

constexpr int kThreads = 128;
constexpr int kKB = 64;                 // k per stage
constexpr uint32_t kLbo = 128;          // bytes between the two 8-wide k halves of a core-matrix pair
constexpr uint32_t kSbo = 1024;         // bytes between 8-row groups (8 k-chunks x 128 B)
constexpr long kWaitLimit = 1L << 22;   // try_wait polls (each suspends briefly): well over a second

__device__ __forceinline__ bool aligned_ptr16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Byte offset of element (r, k) of a 64-wide k block in the canonical layout.
__device__ __forceinline__ uint32_t kmajor_off(int r, int k) {
    return uint32_t(r >> 3) * kSbo + uint32_t(k >> 3) * kLbo + uint32_t(r & 7) * 16u + uint32_t(k & 7) * 2u;
}

// Shared-memory matrix descriptor: start address, LBO, SBO (all >> 4),
// version 1 (sm100), base offset 0, no swizzle.
__device__ __forceinline__ uint64_t smem_desc_lbo_sbo(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return uint64_t((addr >> 4) & 0x3FFFu) | (uint64_t((lbo >> 4) & 0x3FFFu) << 16) |
           (uint64_t((sbo >> 4) & 0x3FFFu) << 32) | (uint64_t(1) << 46);
}
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) { return smem_desc_lbo_sbo(addr, kLbo, kSbo); }

// Instruction descriptor of kind::f16: BF16 A and B (K-major), FP32 D, M = 128.
__host__ __device__ constexpr uint32_t instr_desc(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(n >> 3) << 17) | (uint32_t(128 >> 4) << 24);
}

__device__ __forceinline__ bool mbar_wait(uint32_t addr, uint32_t parity) {
    for (long i = 0; i < kWaitLimit; ++i) {
        uint32_t ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.b32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(addr), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

// tanh(u) = 1 - 2 / (exp(2u) + 1) with the fast exponential (relative error
// ~1e-6, far below the BF16 rounding of the activations it feeds); the
// clamp keeps exp finite.
__device__ __forceinline__ float tanh_fast(float u) {
    const float e = __expf(2.f * fminf(fmaxf(u, -15.f), 15.f));
    return 1.f - __fdividef(2.f, e + 1.f);
}
__device__ __forceinline__ float gelu_f(float x) {
    const float u = 0.7978845608028654f * (x + 0.044715f * x * x * x);
    return 0.5f * x * (1.f + tanh_fast(u));
}
__device__ __forceinline__ float gelu_grad_f(float x) {
    const float u = 0.7978845608028654f * (x + 0.044715f * x * x * x);
    const float t = tanh_fast(u);
    return 0.5f * (1.f + t) + 0.5f * x * (1.f - t * t) * 0.7978845608028654f * (1.f + 3.f * 0.044715f * x * x);
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Copy a (rows x 64) k block (rows valid of nrows_valid, zero beyond) into
// the canonical layout at smem byte address base.
// Loads are issued eight at a time before their stores, so their latencies
// overlap instead of adding up.
__device__ __forceinline__ void load_block(const uint16_t* __restrict__ g, int ld, int row0, int nrows_valid, int k0,
                                           int rows, unsigned char* s) {
    const int chunks = rows * 8;
    for (int c0 = threadIdx.x; c0 < chunks; c0 += 8 * kThreads) {
        uint4 v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int c = c0 + q * kThreads, r = c >> 3, kc = (c & 7) * 8;
            v[q] = make_uint4(0u, 0u, 0u, 0u);
            if (c < chunks && row0 + r < nrows_valid)
                v[q] = *reinterpret_cast<const uint4*>(g + size_t(row0 + r) * ld + k0 + kc);
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int c = c0 + q * kThreads, r = c >> 3, kc = (c & 7) * 8;
            if (c < chunks) *reinterpret_cast<uint4*>(s + kmajor_off(r, kc)) = v[q];
        }
    }
}

// Epilogue: a warp of quarter q (its warp index mod 4, the TMEM lanes it may
// read) reads lanes 32q..32q+31 (rows m0 + 32q + lane of the tile), 16 columns
// at a time from column c_first in steps of c_step, adds the bias, multiplies
// by the GELU derivative of a stored pre-activation (backward), applies GELU,
// and writes the FP32, BF16 and transposed BF16 outputs that are set.
__device__ __forceinline__ void gemm_epilogue(const XpbdGemm& G, uint32_t tmem, int m0, int n0, int n_tile, int warp,
                                              int lane, int c_first = 0, int c_step = 16) {
    const int row = m0 + warp * 32 + lane;
    const bool rv = row < G.m;
    // 16-byte vector stores of a row's 16 columns where the chunk is whole
    // and the row strides keep them aligned
    const bool vec_h = G.out_bf16 && (G.ld_bf16 % 8) == 0 && aligned_ptr16(G.out_bf16);
    const bool vec_f = G.out_f32 && (G.ld_f32 % 4) == 0 && aligned_ptr16(G.out_f32);
    const bool vec_p = G.out_pre && (G.ld_pre % 4) == 0 && aligned_ptr16(G.out_pre);
    for (int c0 = c_first; c0 < n_tile; c0 += c_step) {
        float v[16];
        tmem_ld16(tmem + (uint32_t(warp * 32) << 16) + uint32_t(c0), v);
        if (!rv) continue;
        const bool whole = n0 + c0 + 16 <= G.n;
        float y[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const int col = n0 + c0 + j;
            float z = v[j];
            if (col < G.n) {
                if (G.bias) z += G.bias[col];
                if (G.gelu_grad_of) z *= gelu_grad_f(G.gelu_grad_of[size_t(row) * G.ld_g + col]);
            }
            v[j] = z;
            y[j] = G.act == 1 ? gelu_f(z) : z;
        }
        const size_t cb = size_t(n0 + c0);
        if (G.out_pre) {
            if (whole && vec_p) {
                float4* d = reinterpret_cast<float4*>(G.out_pre + size_t(row) * G.ld_pre + cb);
#pragma unroll
                for (int q = 0; q < 4; ++q) d[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
            } else {
                for (int j = 0; j < 16; ++j)
                    if (n0 + c0 + j < G.n) G.out_pre[size_t(row) * G.ld_pre + cb + j] = v[j];
            }
        }
        if (G.out_f32) {
            if (whole && vec_f) {
                float4* d = reinterpret_cast<float4*>(G.out_f32 + size_t(row) * G.ld_f32 + cb);
#pragma unroll
                for (int q = 0; q < 4; ++q) d[q] = make_float4(y[4 * q], y[4 * q + 1], y[4 * q + 2], y[4 * q + 3]);
            } else {
                for (int j = 0; j < 16; ++j)
                    if (n0 + c0 + j < G.n) G.out_f32[size_t(row) * G.ld_f32 + cb + j] = y[j];
            }
        }
        if (G.out_bf16) {
            __nv_bfloat16* hb = reinterpret_cast<__nv_bfloat16*>(G.out_bf16) + size_t(row) * G.ld_bf16 + cb;
            if (whole && vec_h) {
                uint4 pk[2];
                uint32_t* w = reinterpret_cast<uint32_t*>(pk);
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const __nv_bfloat162 h2 = __floats2bfloat162_rn(y[2 * q], y[2 * q + 1]);
                    w[q] = *reinterpret_cast<const uint32_t*>(&h2);
                }
                reinterpret_cast<uint4*>(hb)[0] = pk[0];
                reinterpret_cast<uint4*>(hb)[1] = pk[1];
            } else {
                for (int j = 0; j < 16; ++j)
                    if (n0 + c0 + j < G.n) hb[j] = __float2bfloat16_rn(y[j]);
            }
        }
        if (G.out_bf16_t) {
            __nv_bfloat16* ht = reinterpret_cast<__nv_bfloat16*>(G.out_bf16_t);
            for (int j = 0; j < 16; ++j)
                if (n0 + c0 + j < G.n) ht[(cb + j) * G.ld_bf16_t + row] = __float2bfloat16_rn(y[j]);
        }
    }
}

__global__ void __launch_bounds__(kThreads, 1) k_gemm_bf16(const __grid_constant__ XpbdGemm G, int n_tile, int tmem_cols) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t s_bar[2];
    __shared__ uint32_t s_tmem;
    const int m0 = blockIdx.x * 128, n0 = blockIdx.y * n_tile;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const size_t a_bytes = size_t(128) * kKB * 2, b_bytes = size_t(n_tile) * kKB * 2;
    unsigned char* sa[2] = {smem, smem + a_bytes + b_bytes};
    unsigned char* sb[2] = {smem + a_bytes, smem + 2 * a_bytes + b_bytes};
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&s_tmem)),
                     "r"(tmem_cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
    }
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&s_bar[0])));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&s_bar[1])));
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = s_tmem;
    const uint32_t idesc = instr_desc(n_tile);
    const int nkb = G.k / kKB;
    bool ok = true;
    for (int kb = 0; kb < nkb && ok; ++kb) {
        const int s = kb & 1;
        if (kb >= 2) ok = mbar_wait(smem_u32(&s_bar[s]), uint32_t(((kb - 2) >> 1) & 1));
        if (!ok) break;
        load_block(G.a, G.lda, m0, G.m, kb * kKB, 128, sa[s]);
        load_block(G.b, G.ldb, n0, G.n, kb * kKB, n_tile, sb[s]);
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const uint32_t a0 = smem_u32(sa[s]), b0 = smem_u32(sb[s]);
#pragma unroll
            for (int ks = 0; ks < kKB / 16; ++ks) {
                const uint64_t ad = smem_desc(a0 + uint32_t(ks) * 2u * kLbo);
                const uint64_t bd = smem_desc(b0 + uint32_t(ks) * 2u * kLbo);
                const uint32_t acc = (kb > 0 || ks > 0) ? 1u : 0u;
                asm volatile(
                    "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                    " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
                    "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                             smem_u32(&s_bar[s]))
                         : "memory");
        }
    }
    if (ok && nkb > 0) ok = mbar_wait(smem_u32(&s_bar[(nkb - 1) & 1]), uint32_t(((nkb - 1) >> 1) & 1));
    if (!ok) {
        if (threadIdx.x == 0 && G.status) atomicOr(G.status, XPBD_STATUS_MMA_TIMEOUT);
        // bounded second wait for the MMAs this CTA issued, then release the tensor memory
        if (nkb > 0) mbar_wait(smem_u32(&s_bar[(nkb - 1) & 1]), uint32_t(((nkb - 1) >> 1) & 1));
    }
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    if (ok) gemm_epilogue(G, tmem, m0, n0, n_tile, warp, lane);
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(tmem_cols));
    }
}

// ---------------------------------------------------------------------------
// The same GEMM with its operands brought in by the tensor memory accelerator.
// A k block of A (128 x 64) and of B (n_tile x 64) is eight 2-D boxes each
// (8 k-elements = 16 bytes wide, 128 or n_tile rows high) that land as
// row-after-row 16-byte lines: eight-row groups are core matrices 128 B apart
// (SBO) and the eight 16-byte k chunks are rows x 16 B apart (LBO).  Rows
// beyond m or n come in as zeros (the tensor map's out-of-bounds fill).  Up to
// kTmaStages k blocks are in flight; one thread issues the copies, waits for
// each block (mbarrier with transaction count), issues its four MMAs and
// commits them to the block's "free" barrier before the stage is refilled.
constexpr int kTmaStages = 4;
// Eight warps: the epilogue (bias, GELU, conversions, stores) is most of the
// kernel's time at the MLP's shapes, and two warps per TMEM lane quarter take
// alternate 16-column chunks.
constexpr int kTmaThreads = 256;

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(
            dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

__global__ void __launch_bounds__(kTmaThreads, 1)
    k_gemm_bf16_tma(const __grid_constant__ XpbdGemm G, const __grid_constant__ CUtensorMap ta,
                    const __grid_constant__ CUtensorMap tb, int n_tile, int tmem_cols) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t s_full[kTmaStages];
    __shared__ __align__(8) uint64_t s_free[kTmaStages];
    __shared__ uint32_t s_tmem;
    __shared__ int s_ok;
    const int m0 = blockIdx.x * 128, n0 = blockIdx.y * n_tile;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t a_lbo = 128u * 16u, b_lbo = uint32_t(n_tile) * 16u;  // bytes per 16-byte k chunk of all rows
    const uint32_t a_bytes = 8u * a_lbo, st_bytes = a_bytes + 8u * b_lbo;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&s_tmem)),
                     "r"(tmem_cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
    }
    if (threadIdx.x == 0) {
        for (int st = 0; st < kTmaStages; ++st) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&s_full[st])));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&s_free[st])));
        }
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        s_ok = 1;
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = s_tmem;
    const int nkb = G.k / kKB;
    if (threadIdx.x == 0) {
        const uint32_t base = smem_u32(smem);
        const uint32_t idesc = instr_desc(n_tile);
        int issued = 0, committed = 0;
        bool ok = true;
        while (issued < nkb && issued < kTmaStages) {
            const int kb = issued++;
            const uint32_t sa = base + uint32_t(kb % kTmaStages) * st_bytes, sb = sa + a_bytes;
            const uint32_t bar = smem_u32(&s_full[kb % kTmaStages]);
            mbar_expect_tx(bar, st_bytes);
            for (int kc = 0; kc < 8; ++kc) {
                tma_load_2d(sa + uint32_t(kc) * a_lbo, &ta, kb * kKB + kc * 8, m0, bar);
                tma_load_2d(sb + uint32_t(kc) * b_lbo, &tb, kb * kKB + kc * 8, n0, bar);
            }
        }
        for (int kb = 0; kb < nkb; ++kb) {
            const int st = kb % kTmaStages;
            const uint32_t par = uint32_t((kb / kTmaStages) & 1);
            if (!mbar_wait(smem_u32(&s_full[st]), par)) {
                ok = false;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const uint32_t sa = base + uint32_t(st) * st_bytes, sb = sa + a_bytes;
#pragma unroll
            for (int ks = 0; ks < kKB / 16; ++ks) {
                const uint64_t ad = smem_desc_lbo_sbo(sa + uint32_t(ks) * 2u * a_lbo, a_lbo, 128u);
                const uint64_t bd = smem_desc_lbo_sbo(sb + uint32_t(ks) * 2u * b_lbo, b_lbo, 128u);
                const uint32_t acc = (kb > 0 || ks > 0) ? 1u : 0u;
                asm volatile(
                    "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                    " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
                    "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                             smem_u32(&s_free[st]))
                         : "memory");
            committed = kb + 1;
            if (issued < nkb) {
                // the stage's next k block may overwrite it only after these MMAs read it
                if (!mbar_wait(smem_u32(&s_free[st]), par)) {
                    ok = false;
                    break;
                }
                const int nk = issued++;
                const uint32_t bar = smem_u32(&s_full[st]);
                mbar_expect_tx(bar, st_bytes);
                for (int kc = 0; kc < 8; ++kc) {
                    tma_load_2d(sa + uint32_t(kc) * a_lbo, &ta, nk * kKB + kc * 8, m0, bar);
                    tma_load_2d(sb + uint32_t(kc) * b_lbo, &tb, nk * kKB + kc * 8, n0, bar);
                }
            }
        }
        // the accumulator is complete when the last commit's barrier completes
        if (ok && committed > 0) {
            const int kl = committed - 1;
            ok = mbar_wait(smem_u32(&s_free[kl % kTmaStages]), uint32_t((kl / kTmaStages) & 1));
        }
        if (!ok) {
            if (G.status) atomicOr(G.status, XPBD_STATUS_MMA_TIMEOUT);
            // bounded waits for this CTA's copies and MMAs still in flight before the
            // shared and tensor memory are released: the last load of every stage, the
            // last commit
            for (int kb = (issued > kTmaStages ? issued - kTmaStages : 0); kb < issued; ++kb)
                mbar_wait(smem_u32(&s_full[kb % kTmaStages]), uint32_t((kb / kTmaStages) & 1));
            if (committed > 0) {
                const int kl = committed - 1;
                mbar_wait(smem_u32(&s_free[kl % kTmaStages]), uint32_t((kl / kTmaStages) & 1));
            }
            s_ok = 0;
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    if (s_ok) gemm_epilogue(G, tmem, m0, n0, n_tile, warp & 3, lane, 16 * (warp >> 2), 32);
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(tmem_cols));
    }
}

// db[o] = sum over valid samples of dzt[o][s] (dzt: transposed BF16 deltas).
__global__ void k_colsum_bf16(int n_out, int m, const uint16_t* __restrict__ dzt, int ld, float* __restrict__ db) {
    const int o = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (o >= n_out) return;
    const __nv_bfloat16* r = reinterpret_cast<const __nv_bfloat16*>(dzt) + size_t(o) * ld;
    float s = 0.f;
    for (int i = lane; i < m; i += 32) s += __bfloat162float(r[i]);
    for (int k = 16; k > 0; k >>= 1) s += __shfl_xor_sync(0xffffffffu, s, k);
    if (lane == 0) db[o] = s;
}

// Adam on FP32 master weights (Kingma & Ba 2015), with the BF16 copy and the
// BF16 transposed copy (rows x cols -> cols x ld_t) refreshed in place.
__global__ void k_adam(int rows, int cols, float* __restrict__ w, const float* __restrict__ g, int ld_g,
                       float* __restrict__ m1, float* __restrict__ m2, float lr, float b1, float b2, float eps,
                       float c1, float c2, uint16_t* __restrict__ wb, uint16_t* __restrict__ wt, int ld_t) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows * cols) return;
    const int r = i / cols, c = i % cols;
    const float gi = g[size_t(r) * ld_g + c];
    const float a = b1 * m1[i] + (1.f - b1) * gi;
    const float b = b2 * m2[i] + (1.f - b2) * gi * gi;
    m1[i] = a;
    m2[i] = b;
    const float wi = w[i] - lr * (a / c1) / (sqrtf(b / c2) + eps);
    w[i] = wi;
    const __nv_bfloat16 h = __float2bfloat16_rn(wi);
    if (wb) reinterpret_cast<__nv_bfloat16*>(wb)[i] = h;
    if (wt) reinterpret_cast<__nv_bfloat16*>(wt)[size_t(c) * ld_t + r] = h;
}

// Loss gradient of the mean squared error over the valid rows:
// d[r][c] = 2 (y - t) / (m * n_out) for r < m, c < n_out; 0 elsewhere in the
// padded (m_pad x ld) BF16 output and its transpose.  loss[0] += sum (y-t)^2.
__global__ void k_mse_grad(int m, int m_pad, int n_out, int ld, const float* __restrict__ y, int ld_y,
                           const float* __restrict__ t, int ld_t, uint16_t* __restrict__ d, uint16_t* __restrict__ dt,
                           int ld_dt, float* __restrict__ loss) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m_pad * ld) return;
    const int r = i / ld, c = i % ld;
    float gval = 0.f;
    if (r < m && c < n_out) {
        const float e = y[size_t(r) * ld_y + c] - t[size_t(r) * ld_t + c];
        gval = 2.f * e / float(m * n_out);
        atomicAdd(loss, e * e);
    }
    const __nv_bfloat16 h = __float2bfloat16_rn(gval);
    reinterpret_cast<__nv_bfloat16*>(d)[i] = h;
    if (dt) reinterpret_cast<__nv_bfloat16*>(dt)[size_t(c) * ld_dt + r] = h;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library); null when the driver does not provide it.
PFN_cuTensorMapEncodeTiled_v12000 encode_tiled() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        cudaGetLastError();
    }
    return fn;
}

// Tensor map of a K-major BF16 operand [rows][ld] (k < ld used): boxes of
// 8 k-elements (16 bytes) x box_rows rows, no swizzle, zero fill outside.
// The caller has checked the 16-byte alignment of the base and of ld x 2.
bool encode_kmajor(CUtensorMap* map, const uint16_t* ptr, int rows, int k, int ld, int box_rows) {
    PFN_cuTensorMapEncodeTiled_v12000 fn = encode_tiled();
    if (!fn || rows <= 0 || k < 8 || box_rows <= 0 || box_rows > 256) return false;
    const cuuint64_t dims[2] = {cuuint64_t(k), cuuint64_t(rows)};
    const cuuint64_t strides[1] = {cuuint64_t(ld) * 2u};
    const cuuint32_t box[2] = {8u, cuuint32_t(box_rows)};
    const cuuint32_t es[2] = {1u, 1u};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<uint16_t*>(ptr), dims, strides, box, es,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

extern "C" {

int xpbd_gemm_bf16(const XpbdGemm* g, int32_t n_tile, xpbd_stream_t stream) {
    if (!g || !g->a || !g->b) return fail(XPBD_ERR_ARG, "xpbd_gemm_bf16: null operand");
    if (g->m <= 0 || g->n <= 0 || g->k <= 0 || g->k % kKB) return fail(XPBD_ERR_ARG, "xpbd_gemm_bf16: m, n > 0, k % 64 == 0");
    if (n_tile < 16 || n_tile > 256 || n_tile % 16) return fail(XPBD_ERR_ARG, "xpbd_gemm_bf16: n_tile in 16..256, % 16");
    if (g->lda < g->k || g->ldb < g->k || g->lda % 8 || g->ldb % 8)
        return fail(XPBD_ERR_ARG, "xpbd_gemm_bf16: lda/ldb >= k and multiples of 8");
    if (!aligned16(g->a) || !aligned16(g->b)) return fail(XPBD_ERR_ALIGN, "xpbd_gemm_bf16: operands 16-byte aligned");
    if (g->act != 0 && g->act != 1) return fail(XPBD_ERR_ARG, "xpbd_gemm_bf16: act");
    int tmem_cols = 32;
    while (tmem_cols < n_tile) tmem_cols <<= 1;
    static bool attr_set[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !attr_set[dev]) {
        if (cudaFuncSetAttribute(k_gemm_bf16, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(size_t(2) * (128 + 256) * kKB * 2)) != cudaSuccess ||
            cudaFuncSetAttribute(k_gemm_bf16_tma, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(size_t(kTmaStages) * (128 + 256) * kKB * 2)) != cudaSuccess)
            return cuda_check("xpbd_gemm_bf16: smem attribute");
        attr_set[dev] = true;
    }
    dim3 grid((g->m + 127) / 128, (g->n + n_tile - 1) / n_tile);
    CUtensorMap ta, tb;
    if (!(g->flags & XPBD_GEMM_THREAD_STAGED) && encode_kmajor(&ta, g->a, g->m, g->k, g->lda, 128) &&
        encode_kmajor(&tb, g->b, g->n, g->k, g->ldb, n_tile)) {
        const size_t smem = size_t(kTmaStages) * (128 + n_tile) * kKB * 2;
        k_gemm_bf16_tma<<<grid, kTmaThreads, smem, (cudaStream_t)stream>>>(*g, ta, tb, n_tile, tmem_cols);
    } else {
        const size_t smem = size_t(2) * (128 + n_tile) * kKB * 2;
        k_gemm_bf16<<<grid, kThreads, smem, (cudaStream_t)stream>>>(*g, n_tile, tmem_cols);
    }
    return cuda_check("xpbd_gemm_bf16");
}

int xpbd_colsum_bf16(int32_t n_out, int32_t m, const uint16_t* dzt, int32_t ld, float* db, xpbd_stream_t stream) {
    if (n_out <= 0 || m <= 0 || !dzt || !db || ld < m) return fail(XPBD_ERR_ARG, "xpbd_colsum_bf16: bad arguments");
    k_colsum_bf16<<<(n_out + 7) / 8, 256, 0, (cudaStream_t)stream>>>(n_out, m, dzt, ld, db);
    return cuda_check("xpbd_colsum_bf16");
}

int xpbd_adam(int32_t rows, int32_t cols, float* w, const float* g, int32_t ld_g, float* m1, float* m2, float lr,
              float beta1, float beta2, float eps, int32_t step, uint16_t* w_bf16, uint16_t* w_bf16_t, int32_t ld_t,
              xpbd_stream_t stream) {
    if (rows <= 0 || cols <= 0 || !w || !g || !m1 || !m2 || step < 1 || ld_g < cols || (w_bf16_t && ld_t < rows))
        return fail(XPBD_ERR_ARG, "xpbd_adam: bad arguments");
    const float c1 = 1.f - powf(beta1, float(step)), c2 = 1.f - powf(beta2, float(step));
    const int n = rows * cols;
    k_adam<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(rows, cols, w, g, ld_g, m1, m2, lr, beta1, beta2, eps,
                                                              c1, c2, w_bf16, w_bf16_t, ld_t);
    return cuda_check("xpbd_adam");
}

int xpbd_mse_grad(int32_t m, int32_t m_pad, int32_t n_out, int32_t ld, const float* y, int32_t ld_y, const float* t,
                  int32_t ld_t, uint16_t* d, uint16_t* d_t, int32_t ld_dt, float* loss, xpbd_stream_t stream) {
    if (m <= 0 || m_pad < m || n_out <= 0 || ld < n_out || !y || !t || !d || !loss || (d_t && ld_dt < m_pad))
        return fail(XPBD_ERR_ARG, "xpbd_mse_grad: bad arguments");
    const int n = m_pad * ld;
    k_mse_grad<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(m, m_pad, n_out, ld, y, ld_y, t, ld_t, d, d_t, ld_dt,
                                                                  loss);
    return cuda_check("xpbd_mse_grad");
}

}  // extern "C"
