// Two-level multigrid transfers between the fine mesh and the coarse cage.
#include <cuda_runtime.h>

#include "xpbd_common.cuh"
#include "xpbd_device.cuh"

using namespace xpbd;

namespace {

constexpr int kMgThreads = 256;

// Fine residual r = x_f - P prior for every embedded fine vertex.
__global__ void __launch_bounds__(kMgThreads)
    k_mg_residual(const __grid_constant__ XpbdCage G, const float4* __restrict__ fine,
                  const float4* __restrict__ coarse) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= G.n_fine) return;
    const int4 id = reinterpret_cast<const int4*>(G.p_idx)[i];
    if (id.x < 0) return;
    const float4 w = reinterpret_cast<const float4*>(G.p_w)[i];
    const float4 a = coarse[id.x], b = coarse[id.y], c = coarse[id.z], d = coarse[id.w];
    const float4 x = fine[i];
    reinterpret_cast<float4*>(G.resid)[i] =
        make_float4(x.x - (((w.x * a.x + w.y * b.x) + w.z * c.x) + w.w * d.x),
                    x.y - (((w.x * a.y + w.y * b.y) + w.z * c.y) + w.w * d.y),
                    x.z - (((w.x * a.z + w.y * b.z) + w.z * c.z) + w.w * d.z), 0.f);
}

// b_c = sum_e w_e r[e] over the restriction CSR of coarse vertex c (cage
// order): one warp per coarse vertex, lanes striding its entries.
__global__ void __launch_bounds__(kMgThreads) k_mg_gather(const __grid_constant__ XpbdCage G) {
    const int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (c >= G.n_coarse) return;
    const float4* res = reinterpret_cast<const float4*>(G.resid);
    float ax = 0.f, ay = 0.f, az = 0.f;
    for (int e = G.r_ptr[c] + lane; e < G.r_ptr[c + 1]; e += 32) {
        const float w = G.r_w[e];
        const float4 x = res[G.r_fine[e]];
        ax += w * x.x;
        ay += w * x.y;
        az += w * x.z;
    }
    for (int o = 16; o > 0; o >>= 1) {
        ax += __shfl_xor_sync(0xffffffffu, ax, o);
        ay += __shfl_xor_sync(0xffffffffu, ay, o);
        az += __shfl_xor_sync(0xffffffffu, az, o);
    }
    if (lane == 0) reinterpret_cast<float4*>(G.rhs)[c] = make_float4(ax, ay, az, 0.f);
}

// Galerkin block solve, kRestrictRows rows of one block per CTA
// (blockIdx.x = block, blockIdx.y = row chunk): the block's right-hand side
// is staged in shared memory, each warp computes rows
// delta[r] = sum_j Minv[r][j] b_j with lanes striding j (coalesced rows) and
// the new coarse position prior + delta.
#ifndef XPBD_RESTRICT_ROWS
#define XPBD_RESTRICT_ROWS 8
#endif
// rows of one block per CTA (one row per warp at 8); every CTA stages the block's
// right-hand side in shared memory, so fewer rows per CTA mean more staging reads
constexpr int kRestrictRows = XPBD_RESTRICT_ROWS;
__global__ void __launch_bounds__(kMgThreads)
    k_mg_restrict(const __grid_constant__ XpbdCage G, float4* coarse, float4* prev, const float4* __restrict__ pin) {
    extern __shared__ float4 sb[];
    const int blk = blockIdx.x;
    const int c0 = G.blk_ptr[blk];
    const int dim = G.blk_ptr[blk + 1] - c0;
    const int r0 = blockIdx.y * kRestrictRows;
    if (r0 >= dim) return;  // uniform over the CTA
    const float4* rhs = reinterpret_cast<const float4*>(G.rhs);
    for (int j = threadIdx.x; j < dim; j += blockDim.x) sb[j] = rhs[c0 + j];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
    const float* M = G.minv + G.blk_moff[blk];
    const int r1 = min(dim, r0 + kRestrictRows);
    for (int r = r0 + warp; r < r1; r += nwarp) {
        const float* row = M + size_t(r) * dim;
        float ax = 0.f, ay = 0.f, az = 0.f;
#pragma unroll 4
        for (int j = lane; j < dim; j += 32) {
            const float m = row[j];
            const float4 b = sb[j];
            ax += m * b.x;
            ay += m * b.y;
            az += m * b.z;
        }
        for (int o = 16; o > 0; o >>= 1) {
            ax += __shfl_xor_sync(0xffffffffu, ax, o);
            ay += __shfl_xor_sync(0xffffffffu, ay, o);
            az += __shfl_xor_sync(0xffffffffu, az, o);
        }
        if (lane == 0) {
            const int cl = G.coarse_lib[c0 + r];
            float4 p = coarse[cl];
            p.x += ax;
            p.y += ay;
            p.z += az;
            if (prev) prev[cl] = make_float4(p.x, p.y, p.z, 0.f);
            if (pin) {
                const float4 t = pin[cl];
                if (t.w != 0.f) {
                    p.x = t.x;
                    p.y = t.y;
                    p.z = t.z;
                }
            }
            coarse[cl] = p;
        }
    }
}

__global__ void __launch_bounds__(kMgThreads)
    k_mg_prolong_delta(const __grid_constant__ XpbdCage G, const float4* __restrict__ coarse,
                       const float4* __restrict__ prev, float4* fine, const int32_t* __restrict__ vflags,
                       const float4* __restrict__ pin) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= G.n_fine) return;
    const int4 id = reinterpret_cast<const int4*>(G.p_idx)[i];
    float4 p = fine[i];
    bool wr = false;
    if (id.x >= 0 && !prev) {  // absolute prolongation (prolong_kernel, mg/kernel.py:181-203)
        const float4 w = reinterpret_cast<const float4*>(G.p_w)[i];
        const float4 a0 = coarse[id.x], a1 = coarse[id.y], a2 = coarse[id.z], a3 = coarse[id.w];
        p.x = ((w.x * a0.x + w.y * a1.x) + w.z * a2.x) + w.w * a3.x;
        p.y = ((w.x * a0.y + w.y * a1.y) + w.z * a2.y) + w.w * a3.y;
        p.z = ((w.x * a0.z + w.y * a1.z) + w.z * a2.z) + w.w * a3.z;
        wr = true;
    } else if (id.x >= 0) {
        const float4 w = reinterpret_cast<const float4*>(G.p_w)[i];
        const float4 a0 = coarse[id.x], b0 = prev[id.x], a1 = coarse[id.y], b1 = prev[id.y];
        const float4 a2 = coarse[id.z], b2 = prev[id.z], a3 = coarse[id.w], b3 = prev[id.w];
        p.x += ((w.x * (a0.x - b0.x) + w.y * (a1.x - b1.x)) + w.z * (a2.x - b2.x)) + w.w * (a3.x - b3.x);
        p.y += ((w.x * (a0.y - b0.y) + w.y * (a1.y - b1.y)) + w.z * (a2.y - b2.y)) + w.w * (a3.y - b3.y);
        p.z += ((w.x * (a0.z - b0.z) + w.y * (a1.z - b1.z)) + w.z * (a2.z - b2.z)) + w.w * (a3.z - b3.z);
        wr = true;
    }
    if (vflags && pin && (vflags[i] & XPBD_VF_PIN)) {
        const float4 t = pin[i];
        if (t.w != 0.f) {
            p.x = t.x;
            p.y = t.y;
            p.z = t.z;
            wr = true;
        }
    }
    if (wr) fine[i] = p;
}

// Step 1 of the V-cycle without the Galerkin restriction (mg_restrict_mode
// "galerkin" / "none", or after the coarse-in-fine readout): the xyz lanes of
// src (when given) replace the coarse position, prev receives the result and
// the coarse kinematic pin overwrites the pinned nodes, as k_mg_restrict does
// after its block solve.  One thread per coarse vertex (library order).
__global__ void __launch_bounds__(kMgThreads)
    k_mg_coarse_reset(int n, const float4* __restrict__ src, float4* coarse, float4* prev,
                      const float4* __restrict__ pin) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 p = coarse[i];
    if (src) {
        const float4 s = src[i];
        p.x = s.x;
        p.y = s.y;
        p.z = s.z;
    }
    if (prev) prev[i] = make_float4(p.x, p.y, p.z, 0.f);
    if (pin) {
        const float4 t = pin[i];
        if (t.w != 0.f) {
            p.x = t.x;
            p.y = t.y;
            p.z = t.z;
        }
    }
    coarse[i] = p;
}

int check_cage(const XpbdCage* g) {
    if (!g || g->n_fine <= 0 || g->n_coarse <= 0 || g->n_blocks <= 0 || !g->r_ptr || !g->r_fine || !g->r_w ||
        !g->blk_ptr || !g->blk_moff || !g->minv || !g->coarse_lib || !g->p_idx || !g->p_w || !g->resid)
        return fail(XPBD_ERR_ARG, "XpbdCage: null member or empty size");
    if (g->max_block <= 0 || g->max_block > 8192) return fail(XPBD_ERR_LIMIT, "XpbdCage: max_block must be in 1..8192");
    if (!g->rhs) return fail(XPBD_ERR_ARG, "XpbdCage: rhs scratch required");
    if (!aligned16(g->p_idx) || !aligned16(g->p_w) || !aligned16(g->resid) || !aligned16(g->rhs))
        return fail(XPBD_ERR_ALIGN, "XpbdCage: p_idx/p_w/resid/rhs alignment");
    return XPBD_OK;
}

}  // namespace

extern "C" {

int xpbd_mg_restrict(const XpbdCage* cage, const float* fine4, float* coarse4, float* coarse_prev4,
                     const float* coarse_pin4, xpbd_stream_t stream) {
    int rc;
    if ((rc = check_cage(cage))) return rc;
    if (!fine4 || !coarse4) return fail(XPBD_ERR_ARG, "xpbd_mg_restrict: null buffer");
    if (!aligned16(fine4) || !aligned16(coarse4) || !aligned16(coarse_prev4) || !aligned16(coarse_pin4))
        return fail(XPBD_ERR_ALIGN, "xpbd_mg_restrict: [n][4] buffers must be 16-byte aligned");
    const size_t smem = size_t(cage->max_block) * sizeof(float4);
    if (smem > kSmemOptIn)
        cudaFuncSetAttribute(k_mg_restrict, cudaFuncAttributeMaxDynamicSharedMemorySize, int(8192 * sizeof(float4)));
    k_mg_residual<<<(cage->n_fine + kMgThreads - 1) / kMgThreads, kMgThreads, 0, (cudaStream_t)stream>>>(
        *cage, reinterpret_cast<const float4*>(fine4), reinterpret_cast<const float4*>(coarse4));
    k_mg_gather<<<(cage->n_coarse * 32 + kMgThreads - 1) / kMgThreads, kMgThreads, 0, (cudaStream_t)stream>>>(*cage);
    const dim3 grid(cage->n_blocks, (cage->max_block + kRestrictRows - 1) / kRestrictRows);
    k_mg_restrict<<<grid, kMgThreads, smem, (cudaStream_t)stream>>>(
        *cage, reinterpret_cast<float4*>(coarse4), reinterpret_cast<float4*>(coarse_prev4),
        reinterpret_cast<const float4*>(coarse_pin4));
    return cuda_check("xpbd_mg_restrict");
}

int xpbd_mg_coarse_reset(const XpbdCage* cage, const float* src4, float* coarse4, float* coarse_prev4,
                         const float* coarse_pin4, xpbd_stream_t stream) {
    int rc;
    if ((rc = check_cage(cage))) return rc;
    if (!coarse4) return fail(XPBD_ERR_ARG, "xpbd_mg_coarse_reset: null coarse buffer");
    if (src4 == coarse4) return fail(XPBD_ERR_ARG, "xpbd_mg_coarse_reset: src4 must not alias coarse4");
    if (!aligned16(src4) || !aligned16(coarse4) || !aligned16(coarse_prev4) || !aligned16(coarse_pin4))
        return fail(XPBD_ERR_ALIGN, "xpbd_mg_coarse_reset: [n][4] buffers must be 16-byte aligned");
    k_mg_coarse_reset<<<(cage->n_coarse + kMgThreads - 1) / kMgThreads, kMgThreads, 0, (cudaStream_t)stream>>>(
        cage->n_coarse, reinterpret_cast<const float4*>(src4), reinterpret_cast<float4*>(coarse4),
        reinterpret_cast<float4*>(coarse_prev4), reinterpret_cast<const float4*>(coarse_pin4));
    return cuda_check("xpbd_mg_coarse_reset");
}

int xpbd_mg_prolong_delta(const XpbdCage* cage, const float* coarse4, const float* coarse_prev4, float* fine4,
                          const int32_t* vflags, const float* pin_target, xpbd_stream_t stream) {
    int rc;
    if ((rc = check_cage(cage))) return rc;
    if (!coarse4 || !fine4) return fail(XPBD_ERR_ARG, "xpbd_mg_prolong_delta: null buffer");
    if (!aligned16(coarse4) || !aligned16(coarse_prev4) || !aligned16(fine4) || !aligned16(pin_target))
        return fail(XPBD_ERR_ALIGN, "xpbd_mg_prolong_delta: [n][4] buffers must be 16-byte aligned");
    k_mg_prolong_delta<<<(cage->n_fine + kMgThreads - 1) / kMgThreads, kMgThreads, 0, (cudaStream_t)stream>>>(
        *cage, reinterpret_cast<const float4*>(coarse4), reinterpret_cast<const float4*>(coarse_prev4),
        reinterpret_cast<float4*>(fine4), vflags, reinterpret_cast<const float4*>(pin_target));
    return cuda_check("xpbd_mg_prolong_delta");
}

}  // extern "C"
