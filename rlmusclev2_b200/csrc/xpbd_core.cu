// Core XPBD substep kernels for sm_100a and their C ABI (include/xpbd_b200.h).
//
// Hot loop per Jacobi iteration: k_project_tiles (one CTA per Morton tile of
// tets: stage the tile's vertices in shared memory, project every constraint
// of every tet, accumulate with shared-memory atomics, apply interior
// vertices in place, push tile-boundary sums to a global float4 accumulator
// with one vector reduction each) followed by k_apply_boundary (finish the
// boundary vertices and clear their accumulator slots).  Between substeps a
// single per-vertex kernel fuses push-out, velocity update, prediction and
// pinning.
#include <cuda_runtime.h>
#include <stdio.h>
#include <cmath>
#include <string.h>

#include "../../include/xpbd_b200.h"
#include "xpbd_common.cuh"
#include "xpbd_device.cuh"
#include "xpbd_tile.cuh"
#include "xpbd_tile_x2.cuh"

using namespace xpbd;

namespace xpbd {
char* err_buffer() {
    static thread_local char buf[256] = "";
    return buf;
}
}  // namespace xpbd

namespace {

constexpr int kTileThreads = 256;
constexpr int kVertThreads = 256;

// L2 prefetch of the bytes [begin, end) of one array through the bulk-copy
// engine: the range is shrunk to whole 16-byte units inside it (the
// instruction wants a 16-byte aligned address and a size in 16-byte units)
// and issued in pieces of at most 32 KB.  A prefetch has no destination and
// no completion to wait for.
__device__ __forceinline__ void prefetch_l2_range(const void* begin, const void* end) {
    uintptr_t a = (reinterpret_cast<uintptr_t>(begin) + 15u) & ~uintptr_t(15);
    const uintptr_t e = reinterpret_cast<uintptr_t>(end) & ~uintptr_t(15);
    while (a < e) {
        const uint32_t n = uint32_t(e - a < 32768u ? e - a : 32768u);
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"(n) : "memory");
        a += n;
    }
}

// The tet streams of one tile: indices and rest matrices, and the fibre
// streams when the tiles carry them.
__device__ __forceinline__ void prefetch_tile_tets(const XpbdTiles& T, int tile) {
    const int t0 = T.tile_tptr[tile], t1 = T.tile_tptr[tile + 1];
    prefetch_l2_range(T.tet_q + 4 * size_t(t0), T.tet_q + 4 * size_t(t1));
    prefetch_l2_range(T.tet_b0 + 4 * size_t(t0), T.tet_b0 + 4 * size_t(t1));
    prefetch_l2_range(T.tet_b1 + 4 * size_t(t0), T.tet_b1 + 4 * size_t(t1));
    prefetch_l2_range(T.tet_b2 + t0, T.tet_b2 + t1);
    if (T.tet_fiber) prefetch_l2_range(T.tet_fiber + 4 * size_t(t0), T.tet_fiber + 4 * size_t(t1));
    if (T.tet_act) prefetch_l2_range(T.tet_act + t0, T.tet_act + t1);
}

template <int MODE, bool DAMP, int MINB, int CSET, bool X2 = false>
__global__ void __launch_bounds__(kTileThreads, MINB)
    k_project_tiles(const __grid_constant__ XpbdParams prm, const __grid_constant__ XpbdTiles T,
                    const __grid_constant__ XpbdVerts V, uint32_t finish_ops) {
    extern __shared__ float4 smem[];
    const int tile = blockIdx.x;
    const int vbeg = T.tile_vptr[tile];
    const int nvt = T.tile_vptr[tile + 1] - vbeg;
    const int nint = (MODE != XPBD_PROJECT_ACCUMULATE) ? T.tile_nint[tile] : 0;
    // Shared layout: positions (float4), previous positions (float4, damped
    // materials only), and the accumulator as four separate 32-bit integer
    // arrays (fixed-point sums, counts) so that atomics on random vertices
    // spread over all 32 banks.
    const int mtv = T.max_tile_verts;
    float4* s_pos = smem;
    float4* s_prev = smem + mtv;
    int* s_ax = reinterpret_cast<int*>(smem + (DAMP ? 2 : 1) * mtv);
    int* s_ay = s_ax + mtv;
    int* s_az = s_ay + mtv;
    int* s_cnt = s_az + mtv;
    const float inv_scale = 1.f / prm.acc_scale;
    const float4* pos4 = reinterpret_cast<const float4*>(V.pos);
    const float4* prev4 = reinterpret_cast<const float4*>(V.pprev);
    __shared__ float s_arap_at[XPBD_MAX_MATERIALS];
    __shared__ int s_defer[2 + kDeferCap];
    // the tet streams are read after the vertex gather: ask for them first
    if ((prm.tile_variant & 32) && threadIdx.x == 0) prefetch_tile_tets(T, tile);
    if (threadIdx.x == 0) s_defer[0] = s_defer[1] = 0;
    fill_arap_at(prm, s_arap_at);
    for (int i = threadIdx.x; i < nvt; i += blockDim.x) {
        const int g = T.tile_verts[vbeg + i];
        s_pos[i] = pos4[g];
        s_ax[i] = 0;
        s_ay[i] = 0;
        s_az[i] = 0;
        s_cnt[i] = 0;
        if (DAMP) s_prev[i] = prev4[g];
    }
    __syncthreads();

    if constexpr (X2 && CSET != CSET_FULL && !DAMP)
        project_tile_tets_x2<CSET == CSET_VOL>(prm, T, tile, s_pos, s_ax, s_ay, s_az, s_cnt, s_arap_at);
    else
        project_tile_tets<DAMP, CSET>(prm, T, tile, s_pos, s_prev, s_ax, s_ay, s_az, s_cnt, s_arap_at, s_defer, 0);
    __syncthreads();

    float4* pos4w = reinterpret_cast<float4*>(V.pos);
    float4* acc4 = reinterpret_cast<float4*>(V.accum);
    if (MODE != XPBD_PROJECT_ACCUMULATE) {
        // Interior vertices: every incident constraint lives in this tile, so
        // the shared sum is complete and no other CTA reads this position.
        for (int i = threadIdx.x; i < nint; i += blockDim.x) {
            const int g = T.tile_verts[vbeg + i];
            float4 pp = s_pos[i];
            finish_vertex(prm, V, g, pp, tile_acc(s_ax, s_ay, s_az, s_cnt, i, inv_scale), finish_ops);
            pos4w[g] = pp;
        }
    }
    for (int i = nint + threadIdx.x; i < nvt; i += blockDim.x) {
        const float4 a = tile_acc(s_ax, s_ay, s_az, s_cnt, i, inv_scale);
        const int g = T.tile_verts[vbeg + i];
        if (MODE != XPBD_PROJECT_FUSED_LAST) {
            if (a.w != 0.f) atomicAdd(&acc4[g], a);
            continue;
        }
        // Every tile touching g adds its partial sum, then counts its arrival;
        // the fence orders the sum before the count.  The tile that arrives
        // last sees all partial sums (fence + L2 load), finishes g from its own
        // staged copy of the old position and resets the slots.  All tiles
        // touching g staged pos[g] before accumulating, so the write cannot be
        // observed by this launch.
        if (a.w != 0.f) atomicAdd(&acc4[g], a);
        __threadfence();
        const int arrived = atomicAdd(&T.arrive[g], 1) + 1;
        if (arrived == T.vert_ntiles[g]) {
            __threadfence();
            const float4 tot = __ldcg(&acc4[g]);
            acc4[g] = make_float4(0.f, 0.f, 0.f, 0.f);
            T.arrive[g] = 0;
            float4 pp = s_pos[i];
            finish_vertex(prm, V, g, pp, tot, finish_ops);
            pos4w[g] = pp;
        }
    }
}

__global__ void __launch_bounds__(kVertThreads)
    k_apply_list(const __grid_constant__ XpbdParams prm, const __grid_constant__ XpbdVerts V, const int32_t* list,
                 int n, uint32_t ops) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int g = list ? list[i] : i;
    float4* acc4 = reinterpret_cast<float4*>(V.accum);
    float4* pos4 = reinterpret_cast<float4*>(V.pos);
    float4 a = make_float4(0.f, 0.f, 0.f, 0.f);
    if (ops & (XPBD_APPLY_ATTACH | XPBD_APPLY_DIVIDE | XPBD_APPLY_CLEAR)) a = acc4[g];
    if (ops & XPBD_APPLY_CLEAR) {
        if (a.x != 0.f || a.y != 0.f || a.z != 0.f || a.w != 0.f) acc4[g] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    float4 p = pos4[g];
    const float4 p0 = p;
    if ((ops & XPBD_APPLY_ATTACH) && !(ops & XPBD_APPLY_DIVIDE)) {
        // accumulate-only: add the ATTACH term to the reference dP/dPw
        const int f = V.vflags ? V.vflags[g] : 0;
        if ((f & XPBD_VF_ATTACH_MASK) && (f & XPBD_VF_ATTACH_MASK) <= prm.n_attach_materials) {
            const XpbdAttachMaterial& M = prm.attach[(f & XPBD_VF_ATTACH_MASK) - 1];
            const float4 at = reinterpret_cast<const float4*>(V.attach_target)[g];
            float3 prev = make_float3(0.f, 0.f, 0.f);
            if (M.damp > 0.f) prev = f3(reinterpret_cast<const float4*>(V.pprev)[g]);
            float3 d;
            if (M.k > 0.f && con_attach(p, prev, f3(at), at.w, M.k, M.damp, prm.dt, d))
                acc4[g] = make_float4(a.x + d.x, a.y + d.y, a.z + d.z, a.w + 1.f);
        }
        return;
    }
    finish_vertex(prm, V, g, p, a, ops);
    if (p.x != p0.x || p.y != p0.y || p.z != p0.z) pos4[g] = p;
}

// ---------------------------------------------------------------------------
// Trilinear grid SDF sample and gradient (phi at nodes origin + h*(i,j,k)).
__device__ __forceinline__ bool sdf_sample(const XpbdSdf& S, float3 x, float& phi, float3& grad) {
    const float inv_h = 1.f / S.h;
    const float gx = (x.x - S.origin[0]) * inv_h, gy = (x.y - S.origin[1]) * inv_h, gz = (x.z - S.origin[2]) * inv_h;
    if (!(gx >= 0.f && gy >= 0.f && gz >= 0.f && gx <= float(S.nx - 1) && gy <= float(S.ny - 1) && gz <= float(S.nz - 1)))
        return false;
    int ix = min(int(gx), S.nx - 2), iy = min(int(gy), S.ny - 2), iz = min(int(gz), S.nz - 2);
    const float fx = gx - float(ix), fy = gy - float(iy), fz = gz - float(iz);
    const size_t sx = 1, sy = size_t(S.nx), sz = size_t(S.nx) * size_t(S.ny);
    const float* b = S.phi + size_t(iz) * sz + size_t(iy) * sy + size_t(ix);
    const float c000 = __ldg(b), c100 = __ldg(b + sx), c010 = __ldg(b + sy), c110 = __ldg(b + sy + sx);
    const float c001 = __ldg(b + sz), c101 = __ldg(b + sz + sx), c011 = __ldg(b + sz + sy), c111 = __ldg(b + sz + sy + sx);
    const float c00 = c000 + fx * (c100 - c000), c10 = c010 + fx * (c110 - c010);
    const float c01 = c001 + fx * (c101 - c001), c11 = c011 + fx * (c111 - c011);
    const float c0 = c00 + fy * (c10 - c00), c1 = c01 + fy * (c11 - c01);
    phi = c0 + fz * (c1 - c0);
    // analytic gradient of the trilinear interpolant
    const float dx0 = (c100 - c000) + fy * ((c110 - c010) - (c100 - c000));
    const float dx1 = (c101 - c001) + fy * ((c111 - c011) - (c101 - c001));
    const float dy0 = (c010 - c000) + fx * ((c110 - c100) - (c010 - c000));
    const float dy1 = (c011 - c001) + fx * ((c111 - c101) - (c011 - c001));
    grad = make_float3((dx0 + fz * (dx1 - dx0)) * inv_h, (dy0 + fz * (dy1 - dy0)) * inv_h, (c1 - c0) * inv_h);
    return true;
}

// Push-out of one vertex (solve_mesh_contact_pos_kernel semantics with the
// bone mesh query replaced by the grid SDF): err = phi - offset; if err < 0
// (and depth <= max_push when max_push > 0) move along the outward normal.
__device__ __forceinline__ void sdf_push(const XpbdSdf& S, float4& p) {
    if (p.w == 0.f) return;
    float phi;
    float3 gr;
    if (!sdf_sample(S, f3(p), phi, gr)) return;
    const float gl = len(gr);
    if (!(gl > 1e-12f)) return;
    const float err = phi - S.contact_offset;
    if (err < 0.f && (S.max_push <= 0.f || -err <= S.max_push)) {
        const float3 n = gr / gl;
        p.x -= n.x * err;
        p.y -= n.y * err;
        p.z -= n.z * err;
    }
}

__device__ __forceinline__ void vertex_step_at(const XpbdParams& prm, const XpbdVerts& V, uint32_t ops,
                                               const XpbdSdf& S, int g) {
    float4* pos4 = reinterpret_cast<float4*>(V.pos);
    float4* prev4 = reinterpret_cast<float4*>(V.pprev);
    float4* vel4 = reinterpret_cast<float4*>(V.vel);
    float4 p = pos4[g];
    float4 v = vel4[g];
    float4 q;
    const float dt = prm.dt;
    if (ops & XPBD_OP_SDF) sdf_push(S, p);
    if (ops & XPBD_OP_VELOCITY) {
        q = prev4[g];
        v.x = (p.x - q.x) / dt;
        v.y = (p.y - q.y) / dt;
        v.z = (p.z - q.z) / dt;
    }
    if (ops & XPBD_OP_PREDICT) {
        q = make_float4(p.x, p.y, p.z, 0.f);
        if (v.w != 0.f) {
            v.x = v.y = v.z = 0.f;
        } else {
            float3 ext = make_float3(prm.gravity[0], prm.gravity[1], prm.gravity[2]);
            const float m = V.mass[g];
            if (V.force && m > 1.0e-12f) ext = ext + f3(reinterpret_cast<const float4*>(V.force)[g]) / m;
            if (prm.quasi_static) {
                const float dt2 = dt * dt;
                p.x += dt2 * ext.x;
                p.y += dt2 * ext.y;
                p.z += dt2 * ext.z;
                v.x = v.y = v.z = 0.f;
            } else {
                const float damp = 1.f - prm.veldamping;
                v.x = damp * v.x + dt * ext.x;
                v.y = damp * v.y + dt * ext.y;
                v.z = damp * v.z + dt * ext.z;
                p.x += dt * v.x;
                p.y += dt * v.y;
                p.z += dt * v.z;
            }
        }
        prev4[g] = q;
    }
    if ((ops & XPBD_OP_PIN) && V.vflags && (V.vflags[g] & XPBD_VF_PIN)) {
        const float4 t = reinterpret_cast<const float4*>(V.pin_target)[g];
        if (t.w != 0.f) {
            p.x = t.x;
            p.y = t.y;
            p.z = t.z;
        }
    }
    pos4[g] = p;
    if (ops & (XPBD_OP_VELOCITY | XPBD_OP_PREDICT)) vel4[g] = v;
}

__global__ void __launch_bounds__(kVertThreads)
    k_vertex_step(const __grid_constant__ XpbdParams prm, const __grid_constant__ XpbdVerts V, uint32_t ops,
                  const __grid_constant__ XpbdSdf S) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= V.n) return;
    vertex_step_at(prm, V, ops, S, g);
}

// Batched instances: each vertex is pushed out of its own instance's grid.
__global__ void __launch_bounds__(kVertThreads)
    k_vertex_step_batched(const __grid_constant__ XpbdParams prm, const __grid_constant__ XpbdVerts V, uint32_t ops,
                          const __grid_constant__ XpbdSdfBatch B) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= V.n) return;
    XpbdSdf S;
    S.nx = B.nx;
    S.ny = B.ny;
    S.nz = B.nz;
    S.contact_offset = B.contact_offset;
    S.max_push = B.max_push;
    S.reserved = 0;
    const int inst = (ops & XPBD_OP_SDF) ? B.vert_inst[g] : -1;
    if (inst >= 0 && inst < B.n_inst) {
        const float4 fr = reinterpret_cast<const float4*>(B.frame)[inst];
        S.phi = B.phi + size_t(inst) * size_t(B.nx) * size_t(B.ny) * size_t(B.nz);
        S.origin[0] = fr.x;
        S.origin[1] = fr.y;
        S.origin[2] = fr.z;
        S.h = fr.w;
    } else {
        S.phi = nullptr;
        S.origin[0] = S.origin[1] = S.origin[2] = 0.f;
        S.h = 1.f;
        ops &= ~uint32_t(XPBD_OP_SDF);
    }
    vertex_step_at(prm, V, ops, S, g);
}

__global__ void k_pin_masked(int n, const int32_t* pts, const float* target, const float* offset,
                             const int32_t* active, float4* pos4) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (active && active[i] == 0) return;
    const int v = pts[i];
    float4 p = pos4[v];
    p.x = target[3 * i] + offset[3 * i];
    p.y = target[3 * i + 1] + offset[3 * i + 1];
    p.z = target[3 * i + 2] + offset[3 * i + 2];
    pos4[v] = p;
}

// ---------------------------------------------------------------------------
// SVD inversion repair (XpbdEngine.repair_inverted_tets, engine.py:831-856):
// per tet with a signed singular value below sigma_min, the edge matrix of
// U diag(max(s, sigma_min)) V^T Dm (Dm = inverse of the rest matrix B, as
// _svd_clamp_accumulate_kernel, engine.py:293-367, computes it), its
// per-vertex difference from the current edges with the centroid kept
// (shift = (d0 + d1 + d2) / 4), added to the Jacobi accumulator of every
// vertex that is not stopped (vel.w == 0) with a count of 1.  Float atomics:
// the repair is a rare correction, not the hot pass.
__device__ __forceinline__ M3 inverse3(const M3& A) {
    M3 C;
    C.m[0][0] = A.m[1][1] * A.m[2][2] - A.m[1][2] * A.m[2][1];
    C.m[0][1] = A.m[0][2] * A.m[2][1] - A.m[0][1] * A.m[2][2];
    C.m[0][2] = A.m[0][1] * A.m[1][2] - A.m[0][2] * A.m[1][1];
    C.m[1][0] = A.m[1][2] * A.m[2][0] - A.m[1][0] * A.m[2][2];
    C.m[1][1] = A.m[0][0] * A.m[2][2] - A.m[0][2] * A.m[2][0];
    C.m[1][2] = A.m[0][2] * A.m[1][0] - A.m[0][0] * A.m[1][2];
    C.m[2][0] = A.m[1][0] * A.m[2][1] - A.m[1][1] * A.m[2][0];
    C.m[2][1] = A.m[0][1] * A.m[2][0] - A.m[0][0] * A.m[2][1];
    C.m[2][2] = A.m[0][0] * A.m[1][1] - A.m[0][1] * A.m[1][0];
    const float d = A.m[0][0] * C.m[0][0] + A.m[0][1] * C.m[1][0] + A.m[0][2] * C.m[2][0];
    const float inv = 1.f / d;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) C.m[i][j] *= inv;
    return C;
}

__global__ void __launch_bounds__(kTileThreads)
    k_svd_clamp(const __grid_constant__ XpbdTiles T, const __grid_constant__ XpbdVerts V, float sigma_min) {
    const int tile = blockIdx.x;
    const int vbeg = T.tile_vptr[tile];
    const float4* pos4 = reinterpret_cast<const float4*>(V.pos);
    const float4* vel4 = reinterpret_cast<const float4*>(V.vel);
    float4* acc = reinterpret_cast<float4*>(V.accum);
    const uint4* tq = reinterpret_cast<const uint4*>(T.tet_q);
    const float4* tb0 = reinterpret_cast<const float4*>(T.tet_b0);
    const float4* tb1 = reinterpret_cast<const float4*>(T.tet_b1);
    for (int t = T.tile_tptr[tile] + threadIdx.x; t < T.tile_tptr[tile + 1]; t += blockDim.x) {
        const uint4 q = tq[t];
        const int g[4] = {T.tile_verts[vbeg + int(q.x & 0xffffu)], T.tile_verts[vbeg + int(q.x >> 16)],
                          T.tile_verts[vbeg + int(q.y & 0xffffu)], T.tile_verts[vbeg + int(q.y >> 16)]};
        const float4 b0 = tb0[t], b1 = tb1[t];
        M3 B;
        B.m[0][0] = b0.x; B.m[0][1] = b0.y; B.m[0][2] = b0.z;
        B.m[1][0] = b0.w; B.m[1][1] = b1.x; B.m[1][2] = b1.y;
        B.m[2][0] = b1.z; B.m[2][1] = b1.w; B.m[2][2] = T.tet_b2[t];
        const float3 p3 = f3(pos4[g[3]]);
        const float3 c[3] = {f3(pos4[g[0]]) - p3, f3(pos4[g[1]]) - p3, f3(pos4[g[2]]) - p3};
        const Svd3 sv = svd3(deformation(c[0], c[1], c[2], B));
        if (sv.s0 >= sigma_min && sv.s1 >= sigma_min && sv.s2 >= sigma_min) continue;
        const float kk[3] = {fmaxf(sv.s0, sigma_min), fmaxf(sv.s1, sigma_min), fmaxf(sv.s2, sigma_min)};
        M3 Ft;  // U diag(clamped s) V^T
        const float U[3][3] = {{sv.u0.x, sv.u1.x, sv.u2.x}, {sv.u0.y, sv.u1.y, sv.u2.y}, {sv.u0.z, sv.u1.z, sv.u2.z}};
        const float W[3][3] = {{sv.v0.x, sv.v1.x, sv.v2.x}, {sv.v0.y, sv.v1.y, sv.v2.y}, {sv.v0.z, sv.v1.z, sv.v2.z}};
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
                Ft.m[i][j] = U[i][0] * kk[0] * W[j][0] + U[i][1] * kk[1] * W[j][1] + U[i][2] * kk[2] * W[j][2];
        const M3 Dm = inverse3(B);
        float3 d[4];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const float3 e = make_float3(Ft.m[0][0] * Dm.m[0][j] + Ft.m[0][1] * Dm.m[1][j] + Ft.m[0][2] * Dm.m[2][j],
                                         Ft.m[1][0] * Dm.m[0][j] + Ft.m[1][1] * Dm.m[1][j] + Ft.m[1][2] * Dm.m[2][j],
                                         Ft.m[2][0] * Dm.m[0][j] + Ft.m[2][1] * Dm.m[1][j] + Ft.m[2][2] * Dm.m[2][j]);
            d[j] = e - c[j];
        }
        const float3 shift = 0.25f * ((d[0] + d[1]) + d[2]);
        d[0] = d[0] - shift;
        d[1] = d[1] - shift;
        d[2] = d[2] - shift;
        d[3] = -shift;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            if (vel4[g[i]].w != 0.f) continue;  // stopped
            float* a = reinterpret_cast<float*>(acc + g[i]);
            atomicAdd(a + 0, d[i].x);
            atomicAdd(a + 1, d[i].y);
            atomicAdd(a + 2, d[i].z);
            atomicAdd(a + 3, 1.f);
        }
    }
}

// _apply_svd_clamp_kernel (engine.py:370-380): pos += alpha dP / w where
// w > 0, then the accumulator is zeroed for the next pass.
__global__ void k_svd_clamp_apply(int n, float4* pos, float4* acc, float alpha) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 a = acc[i];
    if (a.w > 0.f) {
        float4 p = pos[i];
        p.x += (alpha * a.x) / a.w;
        p.y += (alpha * a.y) / a.w;
        p.z += (alpha * a.z) / a.w;
        pos[i] = p;
    }
    acc[i] = make_float4(0.f, 0.f, 0.f, 0.f);
}

// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kTileThreads)
    k_metrics(const __grid_constant__ XpbdTiles T, const __grid_constant__ XpbdVerts V, XpbdMetrics* out) {
    extern __shared__ float4 smem[];
    const int tile = blockIdx.x;
    const int vbeg = T.tile_vptr[tile];
    const int nvt = T.tile_vptr[tile + 1] - vbeg;
    const float4* pos4 = reinterpret_cast<const float4*>(V.pos);
    for (int i = threadIdx.x; i < nvt; i += blockDim.x) smem[i] = pos4[T.tile_verts[vbeg + i]];
    __syncthreads();
    double vol = 0.0, rsq = 0.0;
    float rmax = 0.f;
    int ninv = 0, nnan = 0;
    const uint4* tq = reinterpret_cast<const uint4*>(T.tet_q);
    const float4* tb0 = reinterpret_cast<const float4*>(T.tet_b0);
    const float4* tb1 = reinterpret_cast<const float4*>(T.tet_b1);
    for (int t = T.tile_tptr[tile] + threadIdx.x; t < T.tile_tptr[tile + 1]; t += blockDim.x) {
        const uint4 q = tq[t];
        const float4 b0 = tb0[t], b1 = tb1[t];
        M3 B;
        B.m[0][0] = b0.x; B.m[0][1] = b0.y; B.m[0][2] = b0.z;
        B.m[1][0] = b0.w; B.m[1][1] = b1.x; B.m[1][2] = b1.y;
        B.m[2][0] = b1.z; B.m[2][1] = b1.w; B.m[2][2] = T.tet_b2[t];
        const float3 p0 = f3(smem[q.x & 0xffffu]), p1 = f3(smem[q.x >> 16]), p2 = f3(smem[q.y & 0xffffu]),
                     p3 = f3(smem[q.y >> 16]);
        const float s = p0.x + p0.y + p0.z + p1.x + p1.y + p1.z + p2.x + p2.y + p2.z + p3.x + p3.y + p3.z;
        if (!isfinite(s)) {
            ++nnan;
            continue;
        }
        const M3 F = deformation(p0 - p3, p1 - p3, p2 - p3, B);
        if (det3(F) <= 0.f) ++ninv;
        const float3 d1 = p1 - p0, d2 = p2 - p0, d3 = p3 - p0;
        vol += double(dot(cross(d2, d1), d3) / 6.f);
        const Svd3 sv = svd3(F);
        const float a = sv.s0 - 1.f, b = sv.s1 - 1.f, c = sv.s2 - 1.f;
        const float csq = a * a + b * b + c * c;
        rsq += double(csq);
        rmax = fmaxf(rmax, sqrtf(csq));
    }
    // warp reduce then one atomic per warp
    for (int o = 16; o > 0; o >>= 1) {
        vol += __shfl_down_sync(0xffffffffu, vol, o);
        rsq += __shfl_down_sync(0xffffffffu, rsq, o);
        rmax = fmaxf(rmax, __shfl_down_sync(0xffffffffu, rmax, o));
        ninv += __shfl_down_sync(0xffffffffu, ninv, o);
        nnan += __shfl_down_sync(0xffffffffu, nnan, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&out->vol_sum, vol);
        atomicAdd(&out->resid_sq_sum, rsq);
        atomicMax(reinterpret_cast<int*>(&out->resid_max), __float_as_int(rmax));  // rmax >= 0
        atomicAdd(&out->n_inverted, ninv);
        atomicAdd(&out->n_nonfinite, nnan);
    }
}

int check_verts(const XpbdVerts* v) {
    if (!v || v->n <= 0 || !v->pos) return fail(XPBD_ERR_ARG, "XpbdVerts: null or empty");
    if (!aligned16(v->pos) || !aligned16(v->pprev) || !aligned16(v->vel) || !aligned16(v->accum) ||
        !aligned16(v->force) || !aligned16(v->attach_target) || !aligned16(v->pin_target))
        return fail(XPBD_ERR_ALIGN, "XpbdVerts: a [n][4] array is not 16-byte aligned");
    if (v->vflags && (!v->attach_target || !v->pin_target))
        return fail(XPBD_ERR_ARG, "XpbdVerts: vflags given without attach_target/pin_target");
    return XPBD_OK;
}
int check_params(const XpbdParams* p) {
    if (!p) return fail(XPBD_ERR_ARG, "XpbdParams: null");
    if (p->n_materials < 0 || p->n_materials > XPBD_MAX_MATERIALS || p->n_attach_materials < 0 ||
        p->n_attach_materials > XPBD_MAX_ATTACH_MATERIALS)
        return fail(XPBD_ERR_LIMIT, "XpbdParams: material count out of range");
    if (!(p->dt > 0.f)) return fail(XPBD_ERR_ARG, "XpbdParams: dt must be > 0");
    if (p->tile_variant < 0 || p->tile_variant > 127) return fail(XPBD_ERR_ARG, "XpbdParams: tile_variant must be in 0..127");
    if (!(p->acc_scale > 0.f) || !(p->acc_scale < 3.0e38f))
        return fail(XPBD_ERR_ARG, "XpbdParams: acc_scale must be a finite value > 0 (xpbd_acc_scale_for_extent)");
    return XPBD_OK;
}
int check_tiles(const XpbdTiles* t) {
    if (!t || t->n_tiles <= 0 || !t->tile_vptr || !t->tile_nint || !t->tile_tptr || !t->tile_verts || !t->tet_q ||
        !t->tet_b0 || !t->tet_b1 || !t->tet_b2)
        return fail(XPBD_ERR_ARG, "XpbdTiles: null member");
    if (t->max_tile_verts <= 0 || t->max_tile_verts > XPBD_MAX_TILE_VERTS)
        return fail(XPBD_ERR_LIMIT, "XpbdTiles: max_tile_verts out of range");
    if (!aligned16(t->tet_q) || !aligned16(t->tet_b0) || !aligned16(t->tet_b1) || !aligned16(t->tet_fiber))
        return fail(XPBD_ERR_ALIGN, "XpbdTiles: a [n][4] array is not 16-byte aligned");
    return XPBD_OK;
}

bool any_damped(const XpbdParams* p) {
    for (int i = 0; i < p->n_materials; ++i)
        if (p->materials[i].flags & XPBD_MAT_DAMPED) return true;
    return false;
}
bool any_aniso(const XpbdParams* p) {
    for (int i = 0; i < p->n_materials; ++i)
        if (p->materials[i].flags & XPBD_MAT_ANISO) return true;
    return false;
}

template <int MODE, bool DAMP, int MINB, int CSET, bool X2 = false>
int launch_project_v(const XpbdParams* prm, const XpbdTiles* T, const XpbdVerts* V, uint32_t fops, cudaStream_t s) {
    const size_t smem = size_t(T->max_tile_verts) * sizeof(float4) * (DAMP ? 3 : 2);  // pos, [prev], 4 x float acc
    if (smem > kSmemOptIn) {
        static unsigned char done[64];
        int dev = 0;
        cudaGetDevice(&dev);
        if (dev < 0 || dev >= 64 || !done[dev]) {
            cudaFuncSetAttribute(k_project_tiles<MODE, DAMP, MINB, CSET, X2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(XPBD_MAX_TILE_VERTS * sizeof(float4) * 3));
            if (dev >= 0 && dev < 64) done[dev] = 1;
        }
    }
    k_project_tiles<MODE, DAMP, MINB, CSET, X2><<<T->n_tiles, kTileThreads, smem, s>>>(*prm, *T, *V, fops);
    return cuda_check("xpbd_project");
}

uint32_t material_union(const XpbdParams* p) {
    uint32_t u = 0;
    for (int i = 0; i < p->n_materials; ++i) u |= p->materials[i].flags;
    return u;
}

// Instance choice: the smallest constraint set covering the materials; the
// light set runs 3 CTAs per SM (80 registers, no spills), the others 2 (bit 0
// of tile_variant flips that choice).  Bit 3 runs undamped light and volume
// sets two tets per thread on packed FP32x2 arithmetic (2 CTAs per SM;
// slower on B200, measured: the register pairing costs as many moves as the
// packing saves).
template <int MODE, bool DAMP>
int launch_project(const XpbdParams* prm, const XpbdTiles* T, const XpbdVerts* V, uint32_t fops, cudaStream_t s) {
    const uint32_t u = material_union(prm);
    const bool flip = (prm->tile_variant & 1) != 0;
    if (!DAMP && (prm->tile_variant & 8) && !(u & XPBD_MAT_SNH)) {
        if (u & XPBD_MAT_VOLUME) return launch_project_v<MODE, false, 2, CSET_VOL, true>(prm, T, V, fops, s);
        return launch_project_v<MODE, false, 2, CSET_LIGHT, true>(prm, T, V, fops, s);
    }
    if (u & XPBD_MAT_SNH)
        return flip ? launch_project_v<MODE, DAMP, 3, CSET_FULL>(prm, T, V, fops, s)
                    : launch_project_v<MODE, DAMP, 2, CSET_FULL>(prm, T, V, fops, s);
    if (u & XPBD_MAT_VOLUME)
        return flip ? launch_project_v<MODE, DAMP, 3, CSET_VOL>(prm, T, V, fops, s)
                    : launch_project_v<MODE, DAMP, 2, CSET_VOL>(prm, T, V, fops, s);
    if (DAMP) return launch_project_v<MODE, DAMP, 2, CSET_VOL>(prm, T, V, fops, s);  // damping needs a volume/SNH term
    return flip ? launch_project_v<MODE, false, 2, CSET_LIGHT>(prm, T, V, fops, s)
                : launch_project_v<MODE, false, 3, CSET_LIGHT>(prm, T, V, fops, s);
}

}  // namespace

extern "C" {

int xpbd_abi_version(void) { return 2; }

float xpbd_acc_scale_for_extent(float max_coord) {
    const double e = max_coord > 1e-9f ? double(max_coord) : 1e-9;
    int k = 0;
    while (k < 120 && e * std::ldexp(1.0, k + 1) <= 67108864.0) ++k;
    while (k > -120 && e * std::ldexp(1.0, k) > 67108864.0) --k;
    return float(std::ldexp(1.0, k));
}
const char* xpbd_error_string(void) { return err_buffer(); }

int xpbd_vertex_step(const XpbdParams* prm, const XpbdVerts* v, uint32_t ops, const XpbdSdf* sdf,
                     xpbd_stream_t stream) {
    int rc;
    if ((rc = check_params(prm)) || (rc = check_verts(v))) return rc;
    if ((ops & XPBD_OP_SDF) && (!sdf || !sdf->phi || sdf->nx < 2 || sdf->ny < 2 || sdf->nz < 2 || !(sdf->h > 0.f)))
        return fail(XPBD_ERR_ARG, "xpbd_vertex_step: XPBD_OP_SDF needs a valid XpbdSdf");
    if ((ops & (XPBD_OP_VELOCITY | XPBD_OP_PREDICT)) && (!v->pprev || !v->vel))
        return fail(XPBD_ERR_ARG, "xpbd_vertex_step: pprev/vel required");
    if ((ops & XPBD_OP_PREDICT) && !v->mass) return fail(XPBD_ERR_ARG, "xpbd_vertex_step: mass required");
    XpbdSdf S;
    memset(&S, 0, sizeof(S));
    if (sdf) S = *sdf;
    k_vertex_step<<<(v->n + kVertThreads - 1) / kVertThreads, kVertThreads, 0, (cudaStream_t)stream>>>(*prm, *v, ops, S);
    return cuda_check("xpbd_vertex_step");
}

int xpbd_vertex_step_batched(const XpbdParams* prm, const XpbdVerts* v, uint32_t ops, const XpbdSdfBatch* sdf,
                             xpbd_stream_t stream) {
    int rc;
    if ((rc = check_params(prm)) || (rc = check_verts(v))) return rc;
    if ((ops & XPBD_OP_SDF) && (!sdf || !sdf->phi || !sdf->frame || !sdf->vert_inst || sdf->n_inst < 1 ||
                                sdf->nx < 2 || sdf->ny < 2 || sdf->nz < 2))
        return fail(XPBD_ERR_ARG, "xpbd_vertex_step_batched: XPBD_OP_SDF needs a valid XpbdSdfBatch");
    if ((ops & XPBD_OP_SDF) && !aligned16(sdf->frame)) return fail(XPBD_ERR_ALIGN, "xpbd_vertex_step_batched: frame");
    if ((ops & (XPBD_OP_VELOCITY | XPBD_OP_PREDICT)) && (!v->pprev || !v->vel))
        return fail(XPBD_ERR_ARG, "xpbd_vertex_step_batched: pprev/vel required");
    if ((ops & XPBD_OP_PREDICT) && !v->mass) return fail(XPBD_ERR_ARG, "xpbd_vertex_step_batched: mass required");
    XpbdSdfBatch B;
    memset(&B, 0, sizeof(B));
    if (sdf) B = *sdf;
    k_vertex_step_batched<<<(v->n + kVertThreads - 1) / kVertThreads, kVertThreads, 0, (cudaStream_t)stream>>>(
        *prm, *v, ops, B);
    return cuda_check("xpbd_vertex_step_batched");
}

int xpbd_project(const XpbdParams* prm, const XpbdTiles* tiles, const XpbdVerts* v, int32_t mode,
                 xpbd_stream_t stream) {
    int rc;
    if ((rc = check_params(prm)) || (rc = check_tiles(tiles)) || (rc = check_verts(v))) return rc;
    if (!v->accum) return fail(XPBD_ERR_ARG, "xpbd_project: accum required");
    if (any_aniso(prm) && (!tiles->tet_fiber || !tiles->tet_act))
        return fail(XPBD_ERR_ARG, "xpbd_project: aniso materials need tet_fiber and tet_act");
    const bool damp = any_damped(prm);
    if (damp && !v->pprev) return fail(XPBD_ERR_ARG, "xpbd_project: damped materials need pprev");
    cudaStream_t s = (cudaStream_t)stream;
    const uint32_t fops = XPBD_APPLY_ATTACH | XPBD_APPLY_DIVIDE | XPBD_APPLY_PIN;
    if (mode == XPBD_PROJECT_FUSED)
        return damp ? launch_project<XPBD_PROJECT_FUSED, true>(prm, tiles, v, fops, s)
                    : launch_project<XPBD_PROJECT_FUSED, false>(prm, tiles, v, fops, s);
    if (mode == XPBD_PROJECT_FUSED_LAST) {
        if (!tiles->vert_ntiles || !tiles->arrive)
            return fail(XPBD_ERR_ARG, "xpbd_project: FUSED_LAST needs vert_ntiles and arrive");
        return damp ? launch_project<XPBD_PROJECT_FUSED_LAST, true>(prm, tiles, v, fops, s)
                    : launch_project<XPBD_PROJECT_FUSED_LAST, false>(prm, tiles, v, fops, s);
    }
    if (mode == XPBD_PROJECT_ACCUMULATE)
        return damp ? launch_project<XPBD_PROJECT_ACCUMULATE, true>(prm, tiles, v, 0, s)
                    : launch_project<XPBD_PROJECT_ACCUMULATE, false>(prm, tiles, v, 0, s);
    return fail(XPBD_ERR_ARG, "xpbd_project: unknown mode");
}

int xpbd_apply_boundary(const XpbdParams* prm, const XpbdTiles* tiles, const XpbdVerts* v, uint32_t ops,
                        xpbd_stream_t stream) {
    int rc;
    if ((rc = check_params(prm)) || (rc = check_verts(v))) return rc;
    if (!tiles || (tiles->n_boundary > 0 && !tiles->bnd_verts)) return fail(XPBD_ERR_ARG, "xpbd_apply_boundary: tiles");
    if (!v->accum) return fail(XPBD_ERR_ARG, "xpbd_apply_boundary: accum required");
    if (tiles->n_boundary == 0) return XPBD_OK;
    k_apply_list<<<(tiles->n_boundary + kVertThreads - 1) / kVertThreads, kVertThreads, 0, (cudaStream_t)stream>>>(
        *prm, *v, tiles->bnd_verts, tiles->n_boundary, ops);
    return cuda_check("xpbd_apply_boundary");
}

int xpbd_apply_all(const XpbdParams* prm, const XpbdVerts* v, uint32_t ops, xpbd_stream_t stream) {
    int rc;
    if ((rc = check_params(prm)) || (rc = check_verts(v))) return rc;
    if ((ops & (XPBD_APPLY_ATTACH | XPBD_APPLY_DIVIDE | XPBD_APPLY_CLEAR)) && !v->accum)
        return fail(XPBD_ERR_ARG, "xpbd_apply_all: accum required");
    k_apply_list<<<(v->n + kVertThreads - 1) / kVertThreads, kVertThreads, 0, (cudaStream_t)stream>>>(*prm, *v, nullptr,
                                                                                                       v->n, ops);
    return cuda_check("xpbd_apply_all");
}

int xpbd_pin_overwrite_masked(int32_t n, const int32_t* pts, const float* target, const float* offset,
                              const int32_t* active, float* pos4, xpbd_stream_t stream) {
    if (n < 0 || (n > 0 && (!pts || !target || !offset || !pos4)))
        return fail(XPBD_ERR_ARG, "xpbd_pin_overwrite_masked: bad arguments");
    if (!aligned16(pos4)) return fail(XPBD_ERR_ALIGN, "xpbd_pin_overwrite_masked: pos4 alignment");
    if (n == 0) return XPBD_OK;
    k_pin_masked<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(n, pts, target, offset, active,
                                                                    reinterpret_cast<float4*>(pos4));
    return cuda_check("xpbd_pin_overwrite_masked");
}

int xpbd_metrics(const XpbdTiles* tiles, const XpbdVerts* v, XpbdMetrics* out, xpbd_stream_t stream) {
    int rc;
    if ((rc = check_tiles(tiles)) || (rc = check_verts(v))) return rc;
    if (!out) return fail(XPBD_ERR_ARG, "xpbd_metrics: out");
    cudaStream_t s = (cudaStream_t)stream;
    if (cudaMemsetAsync(out, 0, sizeof(XpbdMetrics), s) != cudaSuccess) return cuda_check("xpbd_metrics memset");
    const size_t smem = size_t(tiles->max_tile_verts) * sizeof(float4);
    if (smem > kSmemOptIn)
        cudaFuncSetAttribute(k_metrics, cudaFuncAttributeMaxDynamicSharedMemorySize, int(XPBD_MAX_TILE_VERTS * sizeof(float4)));
    k_metrics<<<tiles->n_tiles, kTileThreads, smem, s>>>(*tiles, *v, out);
    return cuda_check("xpbd_metrics");
}

int xpbd_svd_clamp(const XpbdTiles* tiles, const XpbdVerts* v, float sigma_min, float alpha, int32_t iters,
                   xpbd_stream_t stream) {
    int rc;
    if ((rc = check_tiles(tiles)) || (rc = check_verts(v))) return rc;
    if (!v->accum || !v->vel) return fail(XPBD_ERR_ARG, "xpbd_svd_clamp: accum and vel required");
    if (!std::isfinite(sigma_min) || !std::isfinite(alpha) || iters < 0)
        return fail(XPBD_ERR_ARG, "xpbd_svd_clamp: finite sigma_min and alpha, iters >= 0");
    if (iters == 0 || alpha <= 0.f) return XPBD_OK;
    cudaStream_t s = (cudaStream_t)stream;
    // clear_dP_kernel before the first pass (engine.py:845-847); each apply pass
    // leaves the accumulator zeroed for the next
    if (cudaMemsetAsync(v->accum, 0, size_t(v->n) * sizeof(float4), s) != cudaSuccess)
        return cuda_check("xpbd_svd_clamp memset");
    for (int it = 0; it < iters; ++it) {
        k_svd_clamp<<<tiles->n_tiles, kTileThreads, 0, s>>>(*tiles, *v, sigma_min);
        k_svd_clamp_apply<<<(v->n + kVertThreads - 1) / kVertThreads, kVertThreads, 0, s>>>(
            v->n, reinterpret_cast<float4*>(v->pos), reinterpret_cast<float4*>(v->accum), alpha);
    }
    return cuda_check("xpbd_svd_clamp");
}

int xpbd_graph_begin(xpbd_stream_t stream) {
    if (cudaStreamBeginCapture((cudaStream_t)stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return cuda_check("xpbd_graph_begin");
    return XPBD_OK;
}
int xpbd_graph_end(xpbd_stream_t stream, void** exec_out) {
    if (!exec_out) return fail(XPBD_ERR_ARG, "xpbd_graph_end: exec_out");
    cudaGraph_t g = nullptr;
    if (cudaStreamEndCapture((cudaStream_t)stream, &g) != cudaSuccess) return cuda_check("xpbd_graph_end");
    cudaGraphExec_t e = nullptr;
    cudaError_t err = cudaGraphInstantiate(&e, g, 0);
    cudaGraphDestroy(g);
    if (err != cudaSuccess) return cuda_check("xpbd_graph_end instantiate");
    *exec_out = e;
    return XPBD_OK;
}
int xpbd_graph_launch(void* exec, xpbd_stream_t stream) {
    if (!exec) return fail(XPBD_ERR_ARG, "xpbd_graph_launch: exec");
    if (cudaGraphLaunch((cudaGraphExec_t)exec, (cudaStream_t)stream) != cudaSuccess)
        return cuda_check("xpbd_graph_launch");
    return XPBD_OK;
}
int xpbd_graph_destroy(void* exec) {
    if (!exec) return XPBD_OK;
    if (cudaGraphExecDestroy((cudaGraphExec_t)exec) != cudaSuccess) return cuda_check("xpbd_graph_destroy");
    return XPBD_OK;
}

}  // extern "C"
