// Per-frame scene kernels: bone-bound vertex targets, grid SDF bake of the
// capsule bones, order permutations.
#include <cuda_runtime.h>
#include <stdio.h>

#include <cmath>

#include "../../include/xpbd_b200.h"
#include "xpbd_common.cuh"
#include "xpbd_device.cuh"

using namespace xpbd;

namespace {

__device__ __forceinline__ float3 xform(const float* T, float4 x) {
    return make_float3(T[0] * x.x + T[1] * x.y + T[2] * x.z + T[3], T[4] * x.x + T[5] * x.y + T[6] * x.z + T[7],
                       T[8] * x.x + T[9] * x.y + T[10] * x.z + T[11]);
}

__global__ void k_bone_targets(int n, int nb, const float* __restrict__ tr, const int2* __restrict__ vb,
                               const float* __restrict__ vw, const float4* __restrict__ rest4, float4* pin, float4* att) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int2 b = vb[i];
    if (b.x < 0 || b.x >= nb || b.y < 0 || b.y >= nb) return;
    const float4 x = rest4[i];
    const float3 ta = xform(tr + 12 * b.x, x);
    float3 t = ta;
    if (vw) {
        const float w = vw[i];
        const float3 tb = xform(tr + 12 * b.y, x);
        t = make_float3(ta.x + w * (tb.x - ta.x), ta.y + w * (tb.y - ta.y), ta.z + w * (tb.z - ta.z));
    }
    if (pin) {
        float4 p = pin[i];
        p.x = t.x; p.y = t.y; p.z = t.z;
        pin[i] = p;
    }
    if (att) {
        float4 a = att[i];
        a.x = t.x; a.y = t.y; a.z = t.z;
        att[i] = a;
    }
}

// pos.xyz += beta (target.xyz - pos.xyz) on vertex v = idx[i] (or i), with
// one rounding per component (fma); indices outside [0, nv) are skipped.
__global__ void k_blend_to_target(int n, const int* __restrict__ idx, int nv, float4* pos,
                                  const float4* __restrict__ tgt, float beta) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int v = idx ? idx[i] : i;
    if (v < 0 || v >= nv) return;
    const float4 t = tgt[v];
    float4 p = pos[v];
    p.x = __fmaf_rn(beta, t.x - p.x, p.x);
    p.y = __fmaf_rn(beta, t.y - p.y, p.y);
    p.z = __fmaf_rn(beta, t.z - p.z, p.z);
    pos[v] = p;
}

constexpr int kBrick = 8;      // 8^3 nodes per CTA
constexpr int kMaxCaps = 256;

struct CapW {
    float3 a, b;  // segment end points (world)
    float r;
};

__device__ __forceinline__ float cap_phi(const CapW& c, float3 x) {
    const float3 ab = c.b - c.a, ax = x - c.a;
    const float L2 = dot(ab, ab);
    const float t = L2 > 0.f ? fminf(fmaxf(dot(ax, ab) / L2, 0.f), 1.f) : 0.f;
    const float3 d = ax - t * ab;
    return len(d) - c.r;
}

// One CTA per 8x8x8 brick of grid nodes: the brick keeps only the capsules
// whose distance to its centre is within band + the brick's half diagonal,
// then every node takes the min over that short list (band elsewhere).
__device__ __forceinline__ void bake_brick(const XpbdSdf& S, int bx, int by, int bz, int nc,
                                           const XpbdCapsule* __restrict__ caps, const float* __restrict__ tr,
                                           float band, CapW* s_cap, int* s_n) {
    if (threadIdx.x == 0) *s_n = 0;
    __syncthreads();
    const float hb = 0.5f * S.h * float(kBrick - 1);
    const float3 bc = make_float3(S.origin[0] + S.h * float(bx * kBrick) + hb, S.origin[1] + S.h * float(by * kBrick) + hb,
                                  S.origin[2] + S.h * float(bz * kBrick) + hb);
    const float brad = hb * 1.7320508f;
    for (int c = threadIdx.x; c < nc; c += blockDim.x) {
        const XpbdCapsule K = caps[c];
        float3 a = make_float3(K.center[0] - K.half * K.axis[0], K.center[1] - K.half * K.axis[1],
                               K.center[2] - K.half * K.axis[2]);
        float3 b = make_float3(K.center[0] + K.half * K.axis[0], K.center[1] + K.half * K.axis[1],
                               K.center[2] + K.half * K.axis[2]);
        if (tr) {
            const float* T = tr + 12 * c;
            const float3 a0 = a, b0 = b;
            a = make_float3(T[0] * a0.x + T[1] * a0.y + T[2] * a0.z + T[3], T[4] * a0.x + T[5] * a0.y + T[6] * a0.z + T[7],
                            T[8] * a0.x + T[9] * a0.y + T[10] * a0.z + T[11]);
            b = make_float3(T[0] * b0.x + T[1] * b0.y + T[2] * b0.z + T[3], T[4] * b0.x + T[5] * b0.y + T[6] * b0.z + T[7],
                            T[8] * b0.x + T[9] * b0.y + T[10] * b0.z + T[11]);
        }
        CapW w{a, b, K.radius};
        if (cap_phi(w, bc) <= band + brad) {
            const int k = atomicAdd(s_n, 1);
            if (k < kMaxCaps) s_cap[k] = w;
        }
    }
    __syncthreads();
    const int ncand = min(*s_n, kMaxCaps);
    const int lx = threadIdx.x & 7, ly = (threadIdx.x >> 3) & 7, lz = threadIdx.x >> 6;
    const int ix = bx * kBrick + lx, iy = by * kBrick + ly, iz = bz * kBrick + lz;
    if (ix >= S.nx || iy >= S.ny || iz >= S.nz) return;
    const float3 x = make_float3(S.origin[0] + S.h * float(ix), S.origin[1] + S.h * float(iy), S.origin[2] + S.h * float(iz));
    float phi = band;
    for (int k = 0; k < ncand; ++k) phi = fminf(phi, cap_phi(s_cap[k], x));
    const_cast<float*>(S.phi)[(size_t(iz) * S.ny + iy) * S.nx + ix] = phi;
}

__global__ void __launch_bounds__(512) k_sdf_bake(const __grid_constant__ XpbdSdf S, int nc,
                                                  const XpbdCapsule* __restrict__ caps,
                                                  const float* __restrict__ tr, float band) {
    __shared__ CapW s_cap[kMaxCaps];
    __shared__ int s_n;
    bake_brick(S, blockIdx.x, blockIdx.y, blockIdx.z, nc, caps, tr, band, s_cap, &s_n);
}

// Batched: blockIdx.z runs over (instance, brick z); instance i bakes its own
// grid from its own capsules caps[i * cpi .. (i + 1) * cpi).
__global__ void __launch_bounds__(512) k_sdf_bake_batched(const __grid_constant__ XpbdSdfBatch B, int cpi,
                                                          const XpbdCapsule* __restrict__ caps,
                                                          const float* __restrict__ tr, float band, int nbz) {
    __shared__ CapW s_cap[kMaxCaps];
    __shared__ int s_n;
    const int inst = blockIdx.z / nbz, bz = blockIdx.z % nbz;
    const float4 fr = reinterpret_cast<const float4*>(B.frame)[inst];
    XpbdSdf S;
    S.phi = B.phi + size_t(inst) * size_t(B.nx) * size_t(B.ny) * size_t(B.nz);
    S.nx = B.nx;
    S.ny = B.ny;
    S.nz = B.nz;
    S.origin[0] = fr.x;
    S.origin[1] = fr.y;
    S.origin[2] = fr.z;
    S.h = fr.w;
    S.contact_offset = B.contact_offset;
    S.max_push = B.max_push;
    S.reserved = 0;
    bake_brick(S, blockIdx.x, blockIdx.y, bz, cpi, caps + size_t(inst) * cpi, tr ? tr + size_t(inst) * cpi * 12 : nullptr,
               band, s_cap, &s_n);
}

__global__ void k_gather(int n, int width, const int32_t* __restrict__ idx, const float* __restrict__ src, int ss,
                         float* __restrict__ dst, int ds) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int j = idx[i];
    for (int c = 0; c < width; ++c) dst[size_t(i) * ds + c] = src[size_t(j) * ss + c];
}

}  // namespace

extern "C" {

int xpbd_bone_targets(int32_t n, int32_t n_bones, const float* transforms, const int32_t* vert_bone,
                      const float* vert_w, const float* rest4, float* pin_target, float* attach_target,
                      xpbd_stream_t stream) {
    if (n < 0 || n_bones <= 0 || !transforms || !vert_bone || !rest4 || (!pin_target && !attach_target))
        return fail(XPBD_ERR_ARG, "xpbd_bone_targets: bad arguments");
    if (!aligned16(rest4) || !aligned16(pin_target) || !aligned16(attach_target) ||
        (reinterpret_cast<uintptr_t>(vert_bone) & 7u))
        return fail(XPBD_ERR_ALIGN, "xpbd_bone_targets: [n][4] arrays must be 16-byte aligned");
    if (n == 0) return XPBD_OK;
    k_bone_targets<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
        n, n_bones, transforms, reinterpret_cast<const int2*>(vert_bone), vert_w, reinterpret_cast<const float4*>(rest4),
        reinterpret_cast<float4*>(pin_target),
        reinterpret_cast<float4*>(attach_target));
    return cuda_check("xpbd_bone_targets");
}

int xpbd_blend_to_target(int32_t n, const int32_t* idx, int32_t n_verts, float* pos4, const float* target4,
                         float beta, xpbd_stream_t stream) {
    if (n < 0 || n_verts < 0 || (!idx && n > n_verts) || (n > 0 && (!pos4 || !target4)) || !std::isfinite(beta))
        return fail(XPBD_ERR_ARG, "xpbd_blend_to_target: bad arguments (finite beta, n <= n_verts without idx)");
    if (!aligned16(pos4) || !aligned16(target4))
        return fail(XPBD_ERR_ALIGN, "xpbd_blend_to_target: [n][4] arrays must be 16-byte aligned");
    if (n == 0 || beta == 0.f) return XPBD_OK;
    k_blend_to_target<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
        n, idx, n_verts, reinterpret_cast<float4*>(pos4), reinterpret_cast<const float4*>(target4), beta);
    return cuda_check("xpbd_blend_to_target");
}

int xpbd_sdf_bake_capsules(const XpbdSdf* sdf, int32_t n_caps, const XpbdCapsule* caps, const float* transforms,
                           float band, xpbd_stream_t stream) {
    if (!sdf || !sdf->phi || sdf->nx < 2 || sdf->ny < 2 || sdf->nz < 2 || !(sdf->h > 0.f) || !(band > 0.f))
        return fail(XPBD_ERR_ARG, "xpbd_sdf_bake_capsules: bad grid");
    if (n_caps < 0 || n_caps > kMaxCaps || (n_caps > 0 && !caps))
        return fail(XPBD_ERR_LIMIT, "xpbd_sdf_bake_capsules: 0 <= n_caps <= 256 required");
    dim3 grid((sdf->nx + kBrick - 1) / kBrick, (sdf->ny + kBrick - 1) / kBrick, (sdf->nz + kBrick - 1) / kBrick);
    k_sdf_bake<<<grid, kBrick * kBrick * kBrick, 0, (cudaStream_t)stream>>>(*sdf, n_caps, caps, transforms, band);
    return cuda_check("xpbd_sdf_bake_capsules");
}

int xpbd_sdf_bake_capsules_batched(const XpbdSdfBatch* sdf, int32_t caps_per_inst, const XpbdCapsule* caps,
                                   const float* transforms, float band, xpbd_stream_t stream) {
    if (!sdf || !sdf->phi || !sdf->frame || sdf->n_inst < 1 || sdf->nx < 2 || sdf->ny < 2 || sdf->nz < 2 ||
        !(band > 0.f))
        return fail(XPBD_ERR_ARG, "xpbd_sdf_bake_capsules_batched: bad grid");
    if (!aligned16(sdf->frame)) return fail(XPBD_ERR_ALIGN, "xpbd_sdf_bake_capsules_batched: frame alignment");
    if (caps_per_inst < 0 || caps_per_inst > kMaxCaps || (caps_per_inst > 0 && !caps))
        return fail(XPBD_ERR_LIMIT, "xpbd_sdf_bake_capsules_batched: 0 <= caps_per_inst <= 256 required");
    const int nbz = (sdf->nz + kBrick - 1) / kBrick;
    if (int64_t(nbz) * sdf->n_inst > 65535) return fail(XPBD_ERR_LIMIT, "xpbd_sdf_bake_capsules_batched: too many grids");
    dim3 grid((sdf->nx + kBrick - 1) / kBrick, (sdf->ny + kBrick - 1) / kBrick, nbz * sdf->n_inst);
    k_sdf_bake_batched<<<grid, kBrick * kBrick * kBrick, 0, (cudaStream_t)stream>>>(*sdf, caps_per_inst, caps,
                                                                                   transforms, band, nbz);
    return cuda_check("xpbd_sdf_bake_capsules_batched");
}

int xpbd_gather(int32_t n, int32_t width, const int32_t* idx, const float* src, int32_t src_stride, float* dst,
                int32_t dst_stride, xpbd_stream_t stream) {
    if (n < 0 || width < 1 || width > 4 || src_stride < width || dst_stride < width || (n > 0 && (!idx || !src || !dst)))
        return fail(XPBD_ERR_ARG, "xpbd_gather: bad arguments");
    if (n == 0) return XPBD_OK;
    k_gather<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(n, width, idx, src, src_stride, dst, dst_stride);
    return cuda_check("xpbd_gather");
}

}  // extern "C"
