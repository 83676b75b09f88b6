// Tile-pass building blocks shared by the per-iteration kernel
// (k_project_tiles, xpbd_core.cu) and the persistent multi-iteration kernel
// (xpbd_persist.cu): the per-vertex finish and the projection of one tile's
// tets into shared-memory accumulators.
#pragma once
#include "xpbd_common.cuh"
#include "xpbd_device.cuh"

namespace xpbd {

// ---------------------------------------------------------------------------
// Per-vertex finish of a Jacobi iteration: ATTACH, divide, pin, from the
// vertex's flags f, attach target at (xyz, restlength), previous position
// (read only for damped attach) and pin target pin (w != 0: active).
__device__ __forceinline__ void finish_core(const XpbdParams& prm, int f, float4 at, float4 prevp, float4 pin, float4& p,
                                            float4 a, uint32_t ops) {
    if ((ops & XPBD_APPLY_ATTACH) && (f & XPBD_VF_ATTACH_MASK) && (f & XPBD_VF_ATTACH_MASK) <= prm.n_attach_materials) {
        const XpbdAttachMaterial& M = prm.attach[(f & XPBD_VF_ATTACH_MASK) - 1];
        if (M.k > 0.f) {
            const float3 prev = M.damp > 0.f ? f3(prevp) : make_float3(0.f, 0.f, 0.f);
            float3 d;
            if (con_attach(p, prev, f3(at), at.w, M.k, M.damp, prm.dt, d)) {
                a.x += d.x;
                a.y += d.y;
                a.z += d.z;
                a.w += 1.f;
            }
        }
    }
    if ((ops & XPBD_APPLY_DIVIDE) && a.w > 1e-9f) {
        float3 d = make_float3(a.x / a.w, a.y / a.w, a.z / a.w);
        if (prm.omega != 1.f) d = prm.omega * d;
        p.x += d.x;
        p.y += d.y;
        p.z += d.z;
    }
    if ((ops & XPBD_APPLY_PIN) && (f & XPBD_VF_PIN) && pin.w != 0.f) {
        p.x = pin.x;
        p.y = pin.y;
        p.z = pin.z;
    }
}

// The finish with the vertex data read from global memory.
__device__ __forceinline__ void finish_vertex(const XpbdParams& prm, const XpbdVerts& V, int g, float4& p, float4 a,
                                              uint32_t ops) {
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    const int f = V.vflags ? V.vflags[g] : 0;
    float4 at = z, prevp = z, pin = z;
    if ((ops & XPBD_APPLY_ATTACH) && (f & XPBD_VF_ATTACH_MASK) && (f & XPBD_VF_ATTACH_MASK) <= prm.n_attach_materials) {
        at = reinterpret_cast<const float4*>(V.attach_target)[g];
        if (prm.attach[(f & XPBD_VF_ATTACH_MASK) - 1].damp > 0.f) prevp = reinterpret_cast<const float4*>(V.pprev)[g];
    }
    if ((ops & XPBD_APPLY_PIN) && (f & XPBD_VF_PIN)) pin = reinterpret_cast<const float4*>(V.pin_target)[g];
    finish_core(prm, f, at, prevp, pin, p, a, ops);
}

// ---------------------------------------------------------------------------
// Per-material ARAP alpha tilde into shared memory (followed by the caller's
// __syncthreads before the first projection).
__device__ __forceinline__ void fill_arap_at(const XpbdParams& prm, float* s_at) {
    for (int i = threadIdx.x; i < prm.n_materials && i < XPBD_MAX_MATERIALS; i += blockDim.x)
        s_at[i] = arap_alpha_tilde(prm.materials[i].arap_k, prm.dt);
}

// ---------------------------------------------------------------------------
// Constraint sets compiled into a tile-pass instance: the heavier sets cost
// registers (and occupancy) even for tets that do not use them.
enum { CSET_LIGHT = 0, CSET_VOL = 1, CSET_FULL = 2 };  // ARAP+aniso | +volume | +volume+SNH

// Projects every constraint of the tile's tets from the staged positions
// (s_pos, s_prev) and adds the Jacobi deltas and counts to the shared
// accumulators s_ax..s_az and the active-constraint counts s_cnt (one
// thread per tet, strided over the CTA).  All four are 32-bit integers added
// with native shared-memory integer atomics (shared float atomics cost about
// five times more): the corrections in fixed point, round(d * acc_scale),
// the counts exactly.  tile_acc reads a vertex's sums back as floats.
__device__ __forceinline__ float4 tile_acc(const int* s_ax, const int* s_ay, const int* s_az, const int* s_cnt, int i,
                                           float inv_scale) {
    return make_float4(float(s_ax[i]) * inv_scale, float(s_ay[i]) * inv_scale, float(s_az[i]) * inv_scale,
                       float(s_cnt[i]));
}

// With tile_variant bit 6, tets whose ARAP rotation needs the SVD (det F <=
// 1e-6 |F|^3: inverted, flat or degenerate; polar_start) are not projected
// where the loop meets them, where a warp would run the SVD with all its
// lanes for one such tet: their ids go to a list in shared memory and, after
// the loop, the CTA projects them together (up to kDeferCap per call; the
// rest are projected in place).  It pays where such tets are common (the
// one-iteration batched boxes: 1.3 % per iteration) and costs 2.6 % where
// they are rare (the 535k-tet muscle scene), so it is off by default.
// A deferred tet runs the same arithmetic as in place (all its constraints,
// the ARAP rotation by the SVD, one rounding of its summed deltas) and the
// integer sums do not depend on the order of the atomics, so the results are
// bit for bit those without the list.  s_defer: two counters and kDeferCap
// ids; call k uses counter k & 1 (parity) and zeroes the other one, so the
// caller zeroes both once before its first call.
constexpr int kDeferCap = 128;

template <bool DAMP, int CSET, bool PREFETCH = false>
__device__ __forceinline__ void project_tile_tets(const XpbdParams& prm, const XpbdTiles& T, int tile,
                                                  const float4* s_pos, const float4* s_prev, int* s_ax, int* s_ay,
                                                  int* s_az, int* s_cnt, const float* s_arap_at,
                                                  int* s_defer = nullptr, int parity = 0) {
    const float acc_scale = prm.acc_scale;
    const float arap_skip = arap_skip_threshold(prm.arap_skip_ssq);
    const bool all_svd = (prm.tile_variant & 2) != 0;
    // uniform over the CTA; tile_variant bit 6 turns the deferred pass on
    const bool defer = s_defer != nullptr && !all_svd && (prm.tile_variant & 64);
    const int t1 = T.tile_tptr[tile + 1];
    const uint4* tq = reinterpret_cast<const uint4*>(T.tet_q);
    const float4* tb0 = reinterpret_cast<const float4*>(T.tet_b0);
    const float4* tb1 = reinterpret_cast<const float4*>(T.tet_b1);
    // One tet from its streams; `late` = the deferred pass.
    auto project_one = [&](int t, const uint4& q, const float4& b0, const float4& b1, float b2, bool late) {
        const int l[4] = {int(q.x & 0xffffu), int(q.x >> 16), int(q.y & 0xffffu), int(q.y >> 16)};
        const XpbdMaterial& m = prm.materials[min(int(q.z & 0xffu), XPBD_MAX_MATERIALS - 1)];
        const float V0 = __uint_as_float(q.w);
        M3 B;
        B.m[0][0] = b0.x; B.m[0][1] = b0.y; B.m[0][2] = b0.z;
        B.m[1][0] = b0.w; B.m[1][1] = b1.x; B.m[1][2] = b1.y;
        B.m[2][0] = b1.z; B.m[2][1] = b1.w; B.m[2][2] = b2;
        float4 p[4], pq[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            p[i] = s_pos[l[i]];
            if (DAMP) pq[i] = s_prev[l[i]];
        }
        const float3 p3 = f3(p[3]);
        const M3 F = deformation(f3(p[0]) - p3, f3(p[1]) - p3, f3(p[2]) - p3, B);
        const uint32_t fl = m.flags;
        if (defer && !late && (fl & XPBD_MAT_ARAPSVD) && !polar_start_ok(F)) {
            const int slot = atomicAdd(s_defer + parity, 1);
            if (slot < kDeferCap) {
                s_defer[2 + slot] = t;
                return;
            }
        }
        // All constraints of the tet read the same positions (Jacobi), so their
        // deltas are summed in registers and pushed with one set of shared
        // atomics; each active constraint adds 1 to dPw of all four vertices.
        float3 d[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) d[i] = make_float3(0.f, 0.f, 0.f);
        int nact = 0;
        // Same type order as the reference table (ascending ConstraintType tag).
        // the deltas arrive already multiplied by acc_scale (a power of two)
        if (CSET >= CSET_FULL && (fl & XPBD_MAT_SNH) &&
            con_snh(p, pq, B, F, V0, m.snh_mu, m.snh_lam, m.snh_damp, prm.dt, acc_scale, d))
            nact += 1;
        if (CSET >= CSET_VOL && (fl & XPBD_MAT_VOLUME) &&
            con_volume(p, pq, V0, m.vol_k, m.vol_damp, prm.dt, acc_scale, d))
            nact += 1;
        if (fl & XPBD_MAT_ANISO) {
            const float4 fb = reinterpret_cast<const float4*>(T.tet_fiber)[t];
            if (con_aniso(p, B, F, f3(fb), fb.w, T.tet_act[t], m.aniso_k, prm.contraction_ratio,
                          prm.fiber_stiffness_scale, prm.dt, acc_scale, d))
                nact += 1;
        }
        if ((fl & XPBD_MAT_ARAPSVD) && con_arapsvd(p, B, F, s_arap_at[min(int(q.z & 0xffu), XPBD_MAX_MATERIALS - 1)],
                                                   arap_skip, acc_scale, d, all_svd || late))
            nact += 1;
        if (nact != 0) {
            // Range check on the sum of the 12 scaled |components| (not their
            // maximum: a sum carries a NaN or Inf component through, fmaxf
            // drops NaN).  Each converted component is then below 2^25 = 2^31/64,
            // so a vertex sum wraps unflagged only with more than 64 such tets on it.
            float dabs = 0.f;
#pragma unroll
            for (int i = 0; i < 4; ++i) dabs += (fabsf(d[i].x) + fabsf(d[i].y)) + fabsf(d[i].z);
            if (!(dabs <= 33554432.f) && prm.status) atomicOr(prm.status, XPBD_STATUS_ACC_RANGE);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                atomicAdd(&s_ax[l[i]], __float2int_rn(d[i].x));
                atomicAdd(&s_ay[l[i]], __float2int_rn(d[i].y));
                atomicAdd(&s_az[l[i]], __float2int_rn(d[i].z));
                atomicAdd(&s_cnt[l[i]], nact);
            }
        }
    };
    // PREFETCH: the next tet's streams are loaded before this tet is
    // projected, so their latency overlaps the math (costs registers).
    int t = T.tile_tptr[tile] + threadIdx.x;
    uint4 qn = make_uint4(0u, 0u, 0u, 0u);
    float4 b0n = make_float4(0.f, 0.f, 0.f, 0.f), b1n = b0n;
    float b2n = 0.f;
    if (PREFETCH && t < t1) {
        qn = tq[t];
        b0n = tb0[t];
        b1n = tb1[t];
        b2n = T.tet_b2[t];
    }
    for (; t < t1; t += blockDim.x) {
        uint4 q;
        float4 b0, b1;
        float b2;
        if (PREFETCH) {
            q = qn;
            b0 = b0n;
            b1 = b1n;
            b2 = b2n;
            const int tn = t + blockDim.x;
            if (tn < t1) {
                qn = tq[tn];
                b0n = tb0[tn];
                b1n = tb1[tn];
                b2n = T.tet_b2[tn];
            }
        } else {
            q = tq[t];
            b0 = tb0[t];
            b1 = tb1[t];
            b2 = T.tet_b2[t];
        }
        project_one(t, q, b0, b1, b2, false);
    }
    if (defer) {
        __syncthreads();
        const int nd = min(s_defer[parity], kDeferCap);
        if (threadIdx.x == 0) s_defer[parity ^ 1] = 0;
        for (int k = threadIdx.x; k < nd; k += blockDim.x) {
            const int td = s_defer[2 + k];
            project_one(td, tq[td], tb0[td], tb1[td], T.tet_b2[td], true);
        }
    }
}

}  // namespace xpbd
