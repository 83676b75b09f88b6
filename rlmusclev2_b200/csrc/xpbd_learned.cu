// Glue kernels of the learned coarse correction: per-cage-vertex features,
// applying the network's correction to the cage, the training target, and the
// residual-gated fallback.  Cage vertices are indexed in cage order j;
// coarse positions live in the coarse engine's library order coarse_lib[j].
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "xpbd_common.cuh"

using namespace xpbd;

namespace {

// Feature row of cage vertex j (64 values):
//  0-2   predicted cage displacement c_pred - c_prev, in mm
//  3     activation of the owning muscle
//  4-12  (R_rel - I) x 10, 13-15 t_rel x 100 (cm): the frame-to-frame motion of
//        the owner's two end bones, blended by the vertex's axial weight
//  16-33 the six lattice neighbours' predicted displacement minus the vertex's (mm; 0 if none)
//  34-36 offset from the rest cage c_pred - c_rest (mm)
//  37-39 offset to the restricted bone-driven targets c_target - c_pred (mm)
//  40-63 static features (rest position in the muscle frame, fiber axis, Fourier terms)
__global__ void k_cage_features(int nc, int m_pad, const int32_t* __restrict__ lib, const float4* __restrict__ cpred,
                                const float4* __restrict__ cprev, const int32_t* __restrict__ nbr,
                                const int32_t* __restrict__ owner, const float* __restrict__ act_muscle,
                                const int2* __restrict__ cbone, const float* __restrict__ cw,
                                const float* __restrict__ bone_rel, const float* __restrict__ stat,
                                const float4* __restrict__ crest, const float4* __restrict__ ctgt,
                                const float* __restrict__ norm, __nv_bfloat16* __restrict__ X,
                                __nv_bfloat16* __restrict__ Xt) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nc) return;
    float f[64];
    const int lj = lib[j];
    const float4 a = cpred[lj], b = cprev[lj];
    const float dx = 1000.f * (a.x - b.x), dy = 1000.f * (a.y - b.y), dz = 1000.f * (a.z - b.z);
    f[0] = dx;
    f[1] = dy;
    f[2] = dz;
    f[3] = act_muscle[owner[j]];
    const int2 bb = cbone[j];
    const float w = cw[j];
    const float* ra = bone_rel + 12 * bb.x;
    const float* rb = bone_rel + 12 * bb.y;
    // blended [R | t] (row-major 3 x 4) of the two end bones' frame-to-frame motion
    float v[12];
#pragma unroll
    for (int i = 0; i < 12; ++i) v[i] = ra[i] + w * (rb[i] - ra[i]);
#pragma unroll
    for (int r = 0; r < 3; ++r) {
#pragma unroll
        for (int c = 0; c < 3; ++c) f[4 + 3 * r + c] = 10.f * (v[4 * r + c] - (r == c ? 1.f : 0.f));
        f[13 + r] = 100.f * v[4 * r + 3];
    }
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        const int k = nbr[6 * j + q];
        float ex = 0.f, ey = 0.f, ez = 0.f;
        if (k >= 0) {
            const int lk = lib[k];
            const float4 ak = cpred[lk], bk = cprev[lk];
            ex = 1000.f * (ak.x - bk.x) - dx;
            ey = 1000.f * (ak.y - bk.y) - dy;
            ez = 1000.f * (ak.z - bk.z) - dz;
        }
        f[16 + 3 * q] = ex;
        f[17 + 3 * q] = ey;
        f[18 + 3 * q] = ez;
    }
    const float4 r0 = crest[lj], tg = ctgt[lj];
    f[34] = 1000.f * (a.x - r0.x);
    f[35] = 1000.f * (a.y - r0.y);
    f[36] = 1000.f * (a.z - r0.z);
    f[37] = 1000.f * (tg.x - a.x);
    f[38] = 1000.f * (tg.y - a.y);
    f[39] = 1000.f * (tg.z - a.z);
#pragma unroll
    for (int i = 0; i < 24; ++i) f[40 + i] = stat[24 * j + i];
#pragma unroll
    for (int i = 0; i < 64; ++i) {
        // standardisation of the training data: (f - mean) / std
        const __nv_bfloat16 h = __float2bfloat16_rn(norm ? (f[i] - norm[2 * i]) * norm[2 * i + 1] : f[i]);
        X[size_t(j) * 64 + i] = h;
        Xt[size_t(i) * m_pad + j] = h;
    }
}

// c_out[lib j].xyz = c_pred[lib j].xyz + scale * y[j][0..2]
__global__ void k_cage_apply(int nc, const int32_t* __restrict__ lib, const float4* __restrict__ cpred,
                             const float* __restrict__ y, int ldy, float scale, float4* __restrict__ cout) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nc) return;
    const int lj = lib[j];
    const float4 a = cpred[lj];
    float4 o = cout[lj];
    o.x = a.x + scale * y[size_t(j) * ldy];
    o.y = a.y + scale * y[size_t(j) * ldy + 1];
    o.z = a.z + scale * y[size_t(j) * ldy + 2];
    cout[lj] = o;
}

// t[j] = scale * (c_star - c_pred)[lib j]
__global__ void k_cage_target(int nc, const int32_t* __restrict__ lib, const float4* __restrict__ cstar,
                              const float4* __restrict__ cpred, float scale, float* __restrict__ t) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nc) return;
    const int lj = lib[j];
    const float4 a = cstar[lj], b = cpred[lj];
    t[3 * j] = scale * (a.x - b.x);
    t[3 * j + 1] = scale * (a.y - b.y);
    t[3 * j + 2] = scale * (a.z - b.z);
}

// Fallback: where the warm-started state's ARAP residual exceeds factor x the
// plain start's (or it has a non-finite position), restore the plain start.
// taken[0] counts fallbacks.
__global__ void k_fallback(int n, const XpbdMetrics* __restrict__ warm, const XpbdMetrics* __restrict__ plain,
                           float factor, const float4* __restrict__ saved, float4* __restrict__ pos, int32_t* taken) {
    const bool back = warm->resid_sq_sum > double(factor) * plain->resid_sq_sum || warm->n_nonfinite > 0;
    if (!back) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0 && taken) atomicAdd(taken, 1);
    if (i < n) pos[i] = saved[i];
}

}  // namespace

extern "C" {

int xpbd_cage_features(const XpbdCageFeatures* cf, const float* c_pred4, const float* c_prev4, uint16_t* X,
                       uint16_t* Xt, xpbd_stream_t stream) {
    if (!cf || !c_pred4 || !c_prev4 || !X || !Xt || cf->n_cage <= 0 || cf->m_pad < cf->n_cage || !cf->coarse_lib ||
        !cf->nbr || !cf->owner || !cf->act_muscle || !cf->cage_bone || !cf->cage_w || !cf->bone_rel || !cf->stat ||
        !cf->c_rest4 || !cf->c_target4)
        return fail(XPBD_ERR_ARG, "xpbd_cage_features: bad arguments");
    if (!aligned16(c_pred4) || !aligned16(c_prev4)) return fail(XPBD_ERR_ALIGN, "xpbd_cage_features: alignment");
    k_cage_features<<<(cf->n_cage + 127) / 128, 128, 0, (cudaStream_t)stream>>>(
        cf->n_cage, cf->m_pad, cf->coarse_lib, reinterpret_cast<const float4*>(c_pred4),
        reinterpret_cast<const float4*>(c_prev4), cf->nbr, cf->owner, cf->act_muscle,
        reinterpret_cast<const int2*>(cf->cage_bone), cf->cage_w, cf->bone_rel, cf->stat,
        reinterpret_cast<const float4*>(cf->c_rest4), reinterpret_cast<const float4*>(cf->c_target4), cf->norm,
        reinterpret_cast<__nv_bfloat16*>(X), reinterpret_cast<__nv_bfloat16*>(Xt));
    return cuda_check("xpbd_cage_features");
}

int xpbd_cage_apply(int32_t n_cage, const int32_t* coarse_lib, const float* c_pred4, const float* y, int32_t ldy,
                    float scale, float* c_out4, xpbd_stream_t stream) {
    if (n_cage <= 0 || !coarse_lib || !c_pred4 || !y || ldy < 3 || !c_out4)
        return fail(XPBD_ERR_ARG, "xpbd_cage_apply: bad arguments");
    k_cage_apply<<<(n_cage + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
        n_cage, coarse_lib, reinterpret_cast<const float4*>(c_pred4), y, ldy, scale, reinterpret_cast<float4*>(c_out4));
    return cuda_check("xpbd_cage_apply");
}

int xpbd_cage_target(int32_t n_cage, const int32_t* coarse_lib, const float* c_star4, const float* c_pred4,
                     float scale, float* t, xpbd_stream_t stream) {
    if (n_cage <= 0 || !coarse_lib || !c_star4 || !c_pred4 || !t) return fail(XPBD_ERR_ARG, "xpbd_cage_target: bad arguments");
    k_cage_target<<<(n_cage + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
        n_cage, coarse_lib, reinterpret_cast<const float4*>(c_star4), reinterpret_cast<const float4*>(c_pred4), scale, t);
    return cuda_check("xpbd_cage_target");
}

int xpbd_fallback_select(int32_t n, const XpbdMetrics* warm, const XpbdMetrics* plain, float factor,
                         const float* saved4, float* pos4, int32_t* taken, xpbd_stream_t stream) {
    if (n <= 0 || !warm || !plain || !saved4 || !pos4 || !(factor > 0.f))
        return fail(XPBD_ERR_ARG, "xpbd_fallback_select: bad arguments");
    k_fallback<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(n, warm, plain, factor,
                                                                  reinterpret_cast<const float4*>(saved4),
                                                                  reinterpret_cast<float4*>(pos4), taken);
    return cuda_check("xpbd_fallback_select");
}

}  // extern "C"
