// Bone-surface binding of muscle vertices: the reference's target_mode="mesh"
// kinematic driver (bone_bind_kernel / bone_slide_target_kernel,
// mg/kernel.py:267-347, driven from mg/mg.py:1117-1174), the per-frame rigid
// pose of capsule bone surfaces, the muscle-to-muscle glue springs
// (solve_m2m_glue_kernel, mg/kernel.py:350-394), and the fascia shell's
// ride coupling to the muscle surface (fascia_bind_kernel /
// fascia_ride_kernel, fascia/fascia.py:130-176).
//
// The reference queries a Warp BVH mesh; here the closest-point query is a
// brute force over the bone faces, staged through shared memory in chunks of
// kFaceChunk faces (the bone surfaces are small next to the muscle mesh, and
// the query runs at bind time and on slide frames only).  One thread per
// muscle vertex.  Barycentric convention of Warp's mesh_eval_position: face
// (A, B, C), position(u, v) = u A + v B + (1 - u - v) C; the face frame is the
// reference's _face_basis (mg/kernel.py:267-285): t1 along position(1,0) -
// position(0,0) = A - C, n the face normal, t2 = n x t1.  Closest point on a
// triangle: the Voronoi-region walk of Ericson, Real-Time Collision Detection
// (2005), sec. 5.1.5; ties between faces keep the lowest face index.
#include <cuda_runtime.h>

#include "xpbd_common.cuh"
#include "xpbd_device.cuh"

using namespace xpbd;

namespace {

constexpr int kBoneThreads = 256;
constexpr int kFaceChunk = 256;

struct FaceFrame {
    float3 t1, t2, n;
};

// squared distance from p to triangle (a, b, c); u, v = weights of a, b
__device__ __forceinline__ float closest_tri(float3 p, float3 a, float3 b, float3 c, float& u, float& v) {
    const float3 ab = b - a, ac = c - a, ap = p - a, bp = p - b, cp = p - c;
    const float d1 = dot(ab, ap), d2 = dot(ac, ap);
    const float d3 = dot(ab, bp), d4 = dot(ac, bp);
    const float d5 = dot(ab, cp), d6 = dot(ac, cp);
    const float vc = d1 * d4 - d3 * d2, vb = d5 * d2 - d1 * d6, va = d3 * d6 - d5 * d4;
    if (d1 <= 0.f && d2 <= 0.f) {
        u = 1.f, v = 0.f;
    } else if (d3 >= 0.f && d4 <= d3) {
        u = 0.f, v = 1.f;
    } else if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f) {
        const float t = d1 / (d1 - d3);
        u = 1.f - t, v = t;
    } else if (d6 >= 0.f && d5 <= d6) {
        u = 0.f, v = 0.f;
    } else if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f) {
        const float t = d2 / (d2 - d6);
        u = 1.f - t, v = 0.f;
    } else if (va <= 0.f && (d4 - d3) >= 0.f && (d5 - d6) >= 0.f) {
        const float t = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        u = 0.f, v = 1.f - t;
    } else {
        const float den = 1.f / (va + vb + vc);
        const float s = vb * den, t = vc * den;
        u = 1.f - s - t, v = s;
    }
    const float w = 1.f - u - v;
    const float3 q = make_float3(u * a.x + v * b.x + w * c.x, u * a.y + v * b.y + w * c.y, u * a.z + v * b.z + w * c.z);
    const float3 e = p - q;
    return dot(e, e);
}

__device__ __forceinline__ void face_corners(const float4* bone, const int* tris, int f, float3& A, float3& B,
                                             float3& C) {
    A = f3(bone[tris[3 * f]]);
    B = f3(bone[tris[3 * f + 1]]);
    C = f3(bone[tris[3 * f + 2]]);
}

__device__ __forceinline__ float3 face_eval(float3 A, float3 B, float3 C, float u, float v) {
    const float w = 1.f - u - v;
    return make_float3(u * A.x + v * B.x + w * C.x, u * A.y + v * B.y + w * C.y, u * A.z + v * B.z + w * C.z);
}

__device__ __forceinline__ float3 unit(float3 a) {
    const float l = sqrtf(dot(a, a));
    const float s = l > 0.f ? 1.f / l : 0.f;
    return make_float3(a.x * s, a.y * s, a.z * s);
}

__device__ __forceinline__ FaceFrame face_frame(float3 A, float3 B, float3 C) {
    // p0 = position(0,0) = C, p1 = position(1,0) = A, p2 = position(0,1) = B
    FaceFrame F;
    F.n = unit(cross(A - C, B - C));
    F.t1 = unit(A - C);
    F.t2 = cross(F.n, F.t1);
    return F;
}

// Closest bone face to p within max_dist (brute force, faces staged in shared
// memory by the whole CTA).  Every thread of the CTA must call it (it holds
// __syncthreads); threads past the query count pass active = false.
__device__ int closest_face(float3 p, bool active, const float4* bone, int nt, const int* tris, float max_dist,
                            float& bu, float& bv, float3 (*s_tri)[3]) {
    int best = -1;
    float bd = max_dist * max_dist;
    for (int f0 = 0; f0 < nt; f0 += kFaceChunk) {
        const int nf = min(kFaceChunk, nt - f0);
        __syncthreads();
        for (int k = threadIdx.x; k < nf; k += blockDim.x)
            face_corners(bone, tris, f0 + k, s_tri[k][0], s_tri[k][1], s_tri[k][2]);
        __syncthreads();
        if (active) {
            for (int k = 0; k < nf; ++k) {
                float u, v;
                const float d = closest_tri(p, s_tri[k][0], s_tri[k][1], s_tri[k][2], u, v);
                if (d < bd || (best < 0 && d <= bd)) {
                    bd = d;
                    best = f0 + k;
                    bu = u;
                    bv = v;
                }
            }
        }
    }
    return best;
}

__device__ __forceinline__ float3 to_local(const FaceFrame& F, float3 d) {
    return make_float3(dot(F.t1, d), dot(F.t2, d), dot(F.n, d));
}

__device__ __forceinline__ float3 from_local(const FaceFrame& F, float4 l) {
    return make_float3(F.t1.x * l.x + F.t2.x * l.y + F.n.x * l.z, F.t1.y * l.x + F.t2.y * l.y + F.n.y * l.z,
                       F.t1.z * l.x + F.t2.z * l.y + F.n.z * l.z);
}

__global__ void __launch_bounds__(kBoneThreads)
    k_bone_bind(int n, const float4* __restrict__ q4, const float4* __restrict__ bone, int nt,
                const int* __restrict__ tris, float max_dist, int* __restrict__ out_face, float2* __restrict__ out_uv,
                float4* __restrict__ out_local) {
    __shared__ float3 s_tri[kFaceChunk][3];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = i < n;
    const float3 p = active ? f3(q4[i]) : make_float3(0.f, 0.f, 0.f);
    float u = 0.f, v = 0.f;
    const int f = closest_face(p, active, bone, nt, tris, max_dist, u, v, s_tri);
    if (!active) return;
    if (f < 0) {  // nothing within max_dist: the reference writes face 0, zero uv and offset
        out_face[i] = 0;
        out_uv[i] = make_float2(0.f, 0.f);
        out_local[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        return;
    }
    float3 A, B, C;
    face_corners(bone, tris, f, A, B, C);
    const float3 cp = face_eval(A, B, C, u, v);
    const float3 l = to_local(face_frame(A, B, C), p - cp);
    out_face[i] = f;
    out_uv[i] = make_float2(u, v);
    out_local[i] = make_float4(l.x, l.y, l.z, 0.f);
}

template <bool REPROJECT>
__global__ void __launch_bounds__(kBoneThreads)
    k_bone_slide_targets(int n, const float4* __restrict__ m4, const int* __restrict__ anchor_face,
                         const float2* __restrict__ anchor_uv, int* __restrict__ bind_face, float2* __restrict__ bind_uv,
                         float4* __restrict__ local4, float slide_range, float max_dist, const float4* __restrict__ bone,
                         int nt, const int* __restrict__ tris, float4* pin_target, float4* attach_target) {
    __shared__ float3 s_tri[REPROJECT ? kFaceChunk : 1][3];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = i < n;
    if (REPROJECT) {
        const float3 p = active ? f3(m4[i]) : make_float3(0.f, 0.f, 0.f);
        float u = 0.f, v = 0.f;
        const int f = closest_face(p, active, bone, nt, tris, max_dist, u, v, s_tri);
        if (active && f >= 0) {
            float3 A, B, C;
            face_corners(bone, tris, anchor_face[i], A, B, C);
            const float2 auv = anchor_uv[i];
            const float3 ap = face_eval(A, B, C, auv.x, auv.y);
            face_corners(bone, tris, f, A, B, C);
            const float3 cand = face_eval(A, B, C, u, v);
            const float3 dd = cand - ap;
            // accept the slide only within slide_range of the leash origin
            if (sqrtf(dot(dd, dd)) <= slide_range) {
                bind_face[i] = f;
                bind_uv[i] = make_float2(u, v);
                const float3 l = to_local(face_frame(A, B, C), p - cand);
                local4[i] = make_float4(l.x, l.y, l.z, 0.f);
            }
        }
    }
    if (!active) return;
    float3 A, B, C;
    const int f = bind_face[i];
    face_corners(bone, tris, f, A, B, C);
    const float2 uv = bind_uv[i];
    const float3 cp = face_eval(A, B, C, uv.x, uv.y);
    const float3 r = from_local(face_frame(A, B, C), local4[i]);
    const float3 t = make_float3(cp.x + r.x, cp.y + r.y, cp.z + r.z);
    if (pin_target) {
        const float4 o = pin_target[i];
        pin_target[i] = make_float4(t.x, t.y, t.z, o.w);
    }
    if (attach_target) {
        const float4 o = attach_target[i];
        attach_target[i] = make_float4(t.x, t.y, t.z, o.w);
    }
}

__global__ void k_bone_surface_pose(int nbv, const float4* __restrict__ rest4, const int* __restrict__ vert_bone,
                                    const float* __restrict__ tr, float4* __restrict__ out4) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nbv) return;
    const float* T = tr + 12 * vert_bone[j];
    const float4 x = rest4[j];
    float o[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) o[r] = ((T[4 * r] * x.x + T[4 * r + 1] * x.y) + T[4 * r + 2] * x.z) + T[4 * r + 3];
    out4[j] = make_float4(o[0], o[1], o[2], 0.f);
}

// solve_m2m_glue_kernel (mg/kernel.py:350-394): one XPBD distance step per
// cross-muscle pair with a fresh multiplier (the reference zeroes L before
// every call), the correction added to both endpoints at once (atomics, as
// the reference's wp.atomic_add).  Inverse masses come from pos4.w (0 for a
// stopped or massless vertex, which then stays put).
__global__ void k_m2m_glue(int n, const int* __restrict__ pa, const int* __restrict__ pb,
                           const float* __restrict__ restlen, const float* __restrict__ compliance, float4* pos4,
                           float dt, float omega) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const int a = pa[c], b = pb[c];
    const float4 xa = pos4[a], xb = pos4[b];
    const float3 d = make_float3(xa.x - xb.x, xa.y - xb.y, xa.z - xb.z);
    const float len = sqrtf(dot(d, d));
    if (len < 1.0e-9f) return;
    const float3 dir = make_float3(d.x / len, d.y / len, d.z / len);
    const float C = len - restlen[c];
    const float wa = xa.w, wb = xb.w;
    const float at = compliance[c] / (dt * dt);
    const float den = (wa + wb) + at;
    if (den < 1.0e-12f) return;
    const float dl = -C / den;
    const float f = omega * dl;
    float* pf = reinterpret_cast<float*>(pos4);
    atomicAdd(pf + 4 * a + 0, (f * wa) * dir.x);
    atomicAdd(pf + 4 * a + 1, (f * wa) * dir.y);
    atomicAdd(pf + 4 * a + 2, (f * wa) * dir.z);
    atomicAdd(pf + 4 * b + 0, (-f * wb) * dir.x);
    atomicAdd(pf + 4 * b + 1, (-f * wb) * dir.y);
    atomicAdd(pf + 4 * b + 2, (-f * wb) * dir.z);
}

// fascia_bind_kernel (fascia/fascia.py:130-157): closest muscle-surface face
// of each fascia rest vertex, its (u, v) and the signed normal gap
// (rest - closest point) . n; ok = 0 when nothing lies within max_dist.
__global__ void __launch_bounds__(kBoneThreads)
    k_surface_bind(int n, const float4* __restrict__ q4, const float4* __restrict__ surf, int nt,
                   const int* __restrict__ tris, float max_dist, int* __restrict__ out_face, float2* __restrict__ out_uv,
                   float* __restrict__ out_gap, int* __restrict__ out_ok) {
    __shared__ float3 s_tri[kFaceChunk][3];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = i < n;
    const float3 p = active ? f3(q4[i]) : make_float3(0.f, 0.f, 0.f);
    float u = 0.f, v = 0.f;
    const int f = closest_face(p, active, surf, nt, tris, max_dist, u, v, s_tri);
    if (!active) return;
    if (f < 0) {
        out_face[i] = 0;
        out_uv[i] = make_float2(0.f, 0.f);
        out_gap[i] = 0.f;
        out_ok[i] = 0;
        return;
    }
    float3 A, B, C;
    face_corners(surf, tris, f, A, B, C);
    const float3 cp = face_eval(A, B, C, u, v);
    out_face[i] = f;
    out_uv[i] = make_float2(u, v);
    out_gap[i] = dot(p - cp, face_frame(A, B, C).n);
    out_ok[i] = 1;
}

// fascia_ride_kernel (fascia/fascia.py:160-176): bound fascia vertex
// bound[i] <- its barycentric point on the current muscle surface + n * gap.
__global__ void k_surface_ride(int n, const int* __restrict__ bound, const int* __restrict__ face,
                               const float2* __restrict__ uv, const float* __restrict__ gap,
                               const float4* __restrict__ surf, const int* __restrict__ tris, float4* fascia4) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float3 A, B, C;
    face_corners(surf, tris, face[i], A, B, C);
    const float2 w = uv[i];
    const float3 cp = face_eval(A, B, C, w.x, w.y);
    const float3 nn = face_frame(A, B, C).n;
    const float g = gap[i];
    const int k = bound[i];
    const float4 o = fascia4[k];
    fascia4[k] = make_float4(cp.x + nn.x * g, cp.y + nn.y * g, cp.z + nn.z * g, o.w);
}

// Fascia squeeze mode (fascia/fascia.py:45-125).  The bone-driven target of
// a muscle vertex is target4[v].xyz (the pin target, target + rest offset).
// fascia_advect_bone_kernel: every shell vertex moves by the frame's change of
// the target of its nearest muscle vertex follow[i].
__global__ void k_fascia_advect(int n, const int* __restrict__ follow, const float4* __restrict__ target4,
                                float4* __restrict__ prev_world, float4* __restrict__ fascia4) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 cur = target4[follow[i]];
    const float4 pw = prev_world[i];
    float4 p = fascia4[i];
    p.x = p.x + (cur.x - pw.x);
    p.y = p.y + (cur.y - pw.y);
    p.z = p.z + (cur.z - pw.z);
    fascia4[i] = p;
    prev_world[i] = make_float4(cur.x, cur.y, cur.z, 0.f);
}

// fascia_anchor_bone_kernel: anchor shell vertices snapped to their muscle
// vertex's bone target plus the rest offset between them.
__global__ void k_fascia_anchor(int n, const int* __restrict__ local, const int* __restrict__ cons,
                                const float4* __restrict__ offset4, const float4* __restrict__ target4,
                                float4* __restrict__ fascia4) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 t = target4[cons[i]], o = offset4[i];
    const int k = local[i];
    const float w = fascia4[k].w;
    fascia4[k] = make_float4(t.x + o.x, t.y + o.y, t.z + o.z, w);
}

// solve_glue_kernel: one-way XPBD distance step from a kinematic shell vertex
// to a muscle vertex (only the muscle moves; fresh multiplier every call),
// atomics on the muscle positions.
__global__ void k_fascia_glue(int n, const int* __restrict__ pf, const int* __restrict__ pm,
                              const float* __restrict__ restlen, const float* __restrict__ compliance,
                              const float4* __restrict__ fascia4, float4* muscle4, float dt, float omega) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const float4 xf = fascia4[pf[c]];
    const int mi = pm[c];
    const float4 xm = muscle4[mi];
    const float3 d = make_float3(xf.x - xm.x, xf.y - xm.y, xf.z - xm.z);
    const float len = sqrtf(dot(d, d));
    if (len < 1.0e-9f) return;
    const float3 dir = make_float3(d.x / len, d.y / len, d.z / len);
    const float C = len - restlen[c];
    const float wj = xm.w;
    const float at = compliance[c] / (dt * dt);
    const float den = wj + at;
    if (den < 1.0e-12f) return;
    const float f = omega * (-C / den);
    float* pm4 = reinterpret_cast<float*>(muscle4) + 4 * mi;
    atomicAdd(pm4 + 0, (-f * wj) * dir.x);
    atomicAdd(pm4 + 1, (-f * wj) * dir.y);
    atomicAdd(pm4 + 2, (-f * wj) * dir.z);
}

bool a16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }
bool a8(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 7u) == 0; }

}  // namespace

extern "C" {

int xpbd_bone_bind(int32_t n, const float* query4, int32_t n_bverts, const float* bone4, int32_t n_btris,
                   const int32_t* btris, float max_dist, int32_t* out_face, float* out_uv, float* out_local4,
                   xpbd_stream_t stream) {
    if (n < 0 || n_bverts <= 0 || n_btris <= 0 || !bone4 || !btris || (n > 0 && (!query4 || !out_face || !out_uv ||
                                                                                  !out_local4)))
        return fail(XPBD_ERR_ARG, "xpbd_bone_bind: bad arguments");
    if (!a16(query4) || !a16(bone4) || !a16(out_local4) || !a8(out_uv))
        return fail(XPBD_ERR_ALIGN, "xpbd_bone_bind: [n][4] arrays 16-byte, uv 8-byte aligned");
    if (n == 0) return XPBD_OK;
    k_bone_bind<<<(n + kBoneThreads - 1) / kBoneThreads, kBoneThreads, 0, (cudaStream_t)stream>>>(
        n, reinterpret_cast<const float4*>(query4), reinterpret_cast<const float4*>(bone4), n_btris, btris, max_dist,
        out_face, reinterpret_cast<float2*>(out_uv), reinterpret_cast<float4*>(out_local4));
    return cuda_check("xpbd_bone_bind");
}

int xpbd_bone_slide_targets(int32_t n, const float* muscle4, const int32_t* anchor_face, const float* anchor_uv,
                            int32_t* bind_face, float* bind_uv, float* local4, float slide_range, int32_t reproject,
                            float max_dist, int32_t n_bverts, const float* bone4, int32_t n_btris,
                            const int32_t* btris, float* pin_target, float* attach_target, xpbd_stream_t stream) {
    if (n < 0 || n_bverts <= 0 || n_btris <= 0 || !bone4 || !btris ||
        (n > 0 && (!bind_face || !bind_uv || !local4 || (!pin_target && !attach_target) ||
                   (reproject && (!muscle4 || !anchor_face || !anchor_uv)))))
        return fail(XPBD_ERR_ARG, "xpbd_bone_slide_targets: bad arguments");
    if (!a16(muscle4) || !a16(bone4) || !a16(local4) || !a16(pin_target) || !a16(attach_target) || !a8(bind_uv) ||
        !a8(anchor_uv))
        return fail(XPBD_ERR_ALIGN, "xpbd_bone_slide_targets: [n][4] arrays 16-byte, uv 8-byte aligned");
    if (n == 0) return XPBD_OK;
    const dim3 grid((n + kBoneThreads - 1) / kBoneThreads);
    cudaStream_t s = (cudaStream_t)stream;
#define XPBD_SLIDE_ARGS                                                                                               \
    n, reinterpret_cast<const float4*>(muscle4), anchor_face, reinterpret_cast<const float2*>(anchor_uv), bind_face, \
        reinterpret_cast<float2*>(bind_uv), reinterpret_cast<float4*>(local4), slide_range, max_dist,               \
        reinterpret_cast<const float4*>(bone4), n_btris, btris, reinterpret_cast<float4*>(pin_target),               \
        reinterpret_cast<float4*>(attach_target)
    if (reproject)
        k_bone_slide_targets<true><<<grid, kBoneThreads, 0, s>>>(XPBD_SLIDE_ARGS);
    else
        k_bone_slide_targets<false><<<grid, kBoneThreads, 0, s>>>(XPBD_SLIDE_ARGS);
#undef XPBD_SLIDE_ARGS
    return cuda_check("xpbd_bone_slide_targets");
}

int xpbd_bone_surface_pose(int32_t n_bverts, const float* rest4, const int32_t* vert_bone, int32_t n_bones,
                           const float* transforms, float* out4, xpbd_stream_t stream) {
    if (n_bverts < 0 || n_bones <= 0 || (n_bverts > 0 && (!rest4 || !vert_bone || !transforms || !out4)))
        return fail(XPBD_ERR_ARG, "xpbd_bone_surface_pose: bad arguments");
    if (!a16(rest4) || !a16(out4)) return fail(XPBD_ERR_ALIGN, "xpbd_bone_surface_pose: [n][4] arrays 16-byte aligned");
    if (n_bverts == 0) return XPBD_OK;
    k_bone_surface_pose<<<(n_bverts + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
        n_bverts, reinterpret_cast<const float4*>(rest4), vert_bone, transforms, reinterpret_cast<float4*>(out4));
    return cuda_check("xpbd_bone_surface_pose");
}

int xpbd_surface_bind(int32_t n, const float* query4, int32_t n_sverts, const float* surf4, int32_t n_stris,
                      const int32_t* stris, float max_dist, int32_t* out_face, float* out_uv, float* out_gap,
                      int32_t* out_ok, xpbd_stream_t stream) {
    if (n < 0 || n_sverts <= 0 || n_stris <= 0 || !surf4 || !stris ||
        (n > 0 && (!query4 || !out_face || !out_uv || !out_gap || !out_ok)))
        return fail(XPBD_ERR_ARG, "xpbd_surface_bind: bad arguments");
    if (!a16(query4) || !a16(surf4) || !a8(out_uv))
        return fail(XPBD_ERR_ALIGN, "xpbd_surface_bind: [n][4] arrays 16-byte, uv 8-byte aligned");
    if (n == 0) return XPBD_OK;
    k_surface_bind<<<(n + kBoneThreads - 1) / kBoneThreads, kBoneThreads, 0, (cudaStream_t)stream>>>(
        n, reinterpret_cast<const float4*>(query4), reinterpret_cast<const float4*>(surf4), n_stris, stris, max_dist,
        out_face, reinterpret_cast<float2*>(out_uv), out_gap, out_ok);
    return cuda_check("xpbd_surface_bind");
}

int xpbd_surface_ride(int32_t n_bound, const int32_t* bound, const int32_t* face, const float* uv, const float* gap,
                      const float* surf4, const int32_t* stris, float* fascia4, xpbd_stream_t stream) {
    if (n_bound < 0 || (n_bound > 0 && (!bound || !face || !uv || !gap || !surf4 || !stris || !fascia4)))
        return fail(XPBD_ERR_ARG, "xpbd_surface_ride: bad arguments");
    if (!a16(surf4) || !a16(fascia4) || !a8(uv))
        return fail(XPBD_ERR_ALIGN, "xpbd_surface_ride: [n][4] arrays 16-byte, uv 8-byte aligned");
    if (n_bound == 0) return XPBD_OK;
    k_surface_ride<<<(n_bound + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
        n_bound, bound, face, reinterpret_cast<const float2*>(uv), gap, reinterpret_cast<const float4*>(surf4), stris,
        reinterpret_cast<float4*>(fascia4));
    return cuda_check("xpbd_surface_ride");
}

int xpbd_fascia_advect(int32_t n, const int32_t* follow, const float* target4, float* prev_world4, float* fascia4,
                       xpbd_stream_t stream) {
    if (n < 0 || (n > 0 && (!follow || !target4 || !prev_world4 || !fascia4)))
        return fail(XPBD_ERR_ARG, "xpbd_fascia_advect: bad arguments");
    if (!a16(target4) || !a16(prev_world4) || !a16(fascia4))
        return fail(XPBD_ERR_ALIGN, "xpbd_fascia_advect: [n][4] arrays must be 16-byte aligned");
    if (n == 0) return XPBD_OK;
    k_fascia_advect<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
        n, follow, reinterpret_cast<const float4*>(target4), reinterpret_cast<float4*>(prev_world4),
        reinterpret_cast<float4*>(fascia4));
    return cuda_check("xpbd_fascia_advect");
}

int xpbd_fascia_anchor(int32_t n, const int32_t* local, const int32_t* cons, const float* offset4,
                       const float* target4, float* fascia4, xpbd_stream_t stream) {
    if (n < 0 || (n > 0 && (!local || !cons || !offset4 || !target4 || !fascia4)))
        return fail(XPBD_ERR_ARG, "xpbd_fascia_anchor: bad arguments");
    if (!a16(offset4) || !a16(target4) || !a16(fascia4))
        return fail(XPBD_ERR_ALIGN, "xpbd_fascia_anchor: [n][4] arrays must be 16-byte aligned");
    if (n == 0) return XPBD_OK;
    k_fascia_anchor<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
        n, local, cons, reinterpret_cast<const float4*>(offset4), reinterpret_cast<const float4*>(target4),
        reinterpret_cast<float4*>(fascia4));
    return cuda_check("xpbd_fascia_anchor");
}

int xpbd_fascia_glue(int32_t n, const int32_t* pair_fascia, const int32_t* pair_muscle, const float* restlen,
                     const float* compliance, const float* fascia4, float* muscle4, float dt, float omega,
                     xpbd_stream_t stream) {
    if (n < 0 || (n > 0 && (!pair_fascia || !pair_muscle || !restlen || !compliance || !fascia4 || !muscle4)) ||
        !(dt > 0.f))
        return fail(XPBD_ERR_ARG, "xpbd_fascia_glue: bad arguments");
    if (!a16(fascia4) || !a16(muscle4))
        return fail(XPBD_ERR_ALIGN, "xpbd_fascia_glue: [n][4] arrays must be 16-byte aligned");
    if (n == 0) return XPBD_OK;
    k_fascia_glue<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
        n, pair_fascia, pair_muscle, restlen, compliance, reinterpret_cast<const float4*>(fascia4),
        reinterpret_cast<float4*>(muscle4), dt, omega);
    return cuda_check("xpbd_fascia_glue");
}

int xpbd_m2m_glue(int32_t n_pairs, const int32_t* pair_a, const int32_t* pair_b, const float* restlen,
                  const float* compliance, float* pos4, float dt, float omega, xpbd_stream_t stream) {
    if (n_pairs < 0 || (n_pairs > 0 && (!pair_a || !pair_b || !restlen || !compliance || !pos4)) || !(dt > 0.f))
        return fail(XPBD_ERR_ARG, "xpbd_m2m_glue: bad arguments");
    if (!a16(pos4)) return fail(XPBD_ERR_ALIGN, "xpbd_m2m_glue: pos4 must be 16-byte aligned");
    if (n_pairs == 0) return XPBD_OK;
    k_m2m_glue<<<(n_pairs + 255) / 256, 256, 0, (cudaStream_t)stream>>>(n_pairs, pair_a, pair_b, restlen, compliance,
                                                                        reinterpret_cast<float4*>(pos4), dt, omega);
    return cuda_check("xpbd_m2m_glue");
}

}  // extern "C"
