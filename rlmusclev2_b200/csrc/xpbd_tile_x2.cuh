// Two-tet packed projection of the ARAP-SVD / aniso_arap constraint set.
//
// Blackwell executes FP32 add, multiply and fused multiply-add on pairs of
// values held in a 64-bit register pair (__fadd2_rn, __fmul2_rn, __ffma2_rn:
// one instruction, two IEEE-rounded results, each bit-identical to the
// scalar operation).  The tile pass is bound by instruction issue, so each
// thread projects two tets at once with every FP32 step of the ARAP-SVD
// constraint -- the deformation gradient, the polar iteration, the gradient
// rows, the Lagrange step -- written on (tet a, tet b) pairs.  Transcendental
// steps (power, reciprocal, reciprocal square root), the rare SVD fallback of
// inverted tets, the aniso_arap term of the one aniso muscle and the
// fixed-point shared-memory accumulation stay per tet.
//
// Same arithmetic as con_arapsvd (xpbd_device.cuh) in the same order, with
// two differences of a few ulps: the ARAP step dL = -C / (w + alpha~) uses
// the fast reciprocal, and C = ssq * rsqrt(ssq).  A tet whose rotation needs
// more Newton steps than its partner keeps iterating until both converge (the
// converged one then stays at its fixed point).
#pragma once
#include <cuda_runtime.h>

#include "xpbd_common.cuh"
#include "xpbd_device.cuh"
#include "xpbd_tile.cuh"

namespace xpbd {

typedef float2 f2;

__device__ __forceinline__ f2 pk(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ f2 add2(f2 a, f2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ f2 mul2(f2 a, f2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ f2 neg2(f2 a) { return make_float2(-a.x, -a.y); }
// a - b with one rounding, as the scalar subtraction
__device__ __forceinline__ f2 sub2(f2 a, f2 b) { return __ffma2_rn(make_float2(-1.f, -1.f), b, a); }

struct V2 {
    f2 x, y, z;
};

__device__ __forceinline__ V2 vsub2(const V2& a, const V2& b) { return {sub2(a.x, b.x), sub2(a.y, b.y), sub2(a.z, b.z)}; }
__device__ __forceinline__ f2 vdot2(const V2& a, const V2& b) { return fma2(a.z, b.z, fma2(a.y, b.y, mul2(a.x, b.x))); }
// a x b, each component a.y*b.z - a.z*b.y as fma(a.y, b.z, -(a.z*b.y))
__device__ __forceinline__ V2 vcross2(const V2& a, const V2& b) {
    return {fma2(a.y, b.z, neg2(mul2(a.z, b.y))), fma2(a.z, b.x, neg2(mul2(a.x, b.z))),
            fma2(a.x, b.y, neg2(mul2(a.y, b.x)))};
}
// s * a + t * c
__device__ __forceinline__ V2 vaxpy2(f2 s, const V2& a, f2 t, const V2& c) {
    return {fma2(t, c.x, mul2(s, a.x)), fma2(t, c.y, mul2(s, a.y)), fma2(t, c.z, mul2(s, a.z))};
}

// One scaled Newton step X <- g X / 2 + (g X)^-T / 2 on the columns of both
// tets' X (Higham's scaled Newton step, per lane).  c0 = x1 x x2 and
// det = x0 . c0 come in; the new columns overwrite x0..x2 and the squared
// step norm is returned.
__device__ __forceinline__ f2 polar_step2(V2& x0, V2& x1, V2& x2, const V2& c0, f2 det) {
    const V2 c1 = vcross2(x2, x0), c2 = vcross2(x0, x1);
    const float ga = __powf(det.x, -0.33333334f), gb = __powf(det.y, -0.33333334f);
    const f2 g = pk(ga, gb);
    const f2 gd = mul2(g, det);
    const f2 h = pk(__fdividef(0.5f, gd.x), __fdividef(0.5f, gd.y));
    const f2 a = mul2(pk(0.5f, 0.5f), g);
    const V2 y0 = vaxpy2(a, x0, h, c0), y1 = vaxpy2(a, x1, h, c1), y2 = vaxpy2(a, x2, h, c2);
    const V2 e0 = vsub2(y0, x0), e1 = vsub2(y1, x1), e2 = vsub2(y2, x2);
    const f2 ch = add2(add2(vdot2(e0, e0), vdot2(e1, e1)), vdot2(e2, e2));
    x0 = y0;
    x1 = y1;
    x2 = y2;
    return ch;
}

// Rotation of the polar decomposition F = R S of both tets (columns of F in
// x0..x2 on entry, of R on exit), Higham's scaled Newton iteration as
// polar_rotation (xpbd_device.cuh).  ok.x / ok.y: false where that tet needs
// the SVD (det F <= 1e-6 |F|^3, a non-positive determinant on the way, or no
// convergence in 10 steps).
__device__ __forceinline__ void polar_rotation2(V2& x0, V2& x1, V2& x2, bool& oka, bool& okb) {
    const f2 n2 = add2(add2(vdot2(x0, x0), vdot2(x1, x1)), vdot2(x2, x2));
    V2 c0 = vcross2(x1, x2);
    f2 det = vdot2(x0, c0);
    oka = det.x > 0.f && det.x * det.x > 1e-12f * (n2.x * n2.x * n2.x);
    okb = det.y > 0.f && det.y * det.y > 1e-12f * (n2.y * n2.y * n2.y);
    if (!oka && !okb) return;
    // a failed lane iterates on a harmless stand-in (the identity) so the pair stays packed
    if (!oka) {
        x0.x.x = 1.f; x0.y.x = 0.f; x0.z.x = 0.f; x1.x.x = 0.f; x1.y.x = 1.f; x1.z.x = 0.f;
        x2.x.x = 0.f; x2.y.x = 0.f; x2.z.x = 1.f; c0.x.x = 1.f; c0.y.x = 0.f; c0.z.x = 0.f; det.x = 1.f;
    }
    if (!okb) {
        x0.x.y = 1.f; x0.y.y = 0.f; x0.z.y = 0.f; x1.x.y = 0.f; x1.y.y = 1.f; x1.z.y = 0.f;
        x2.x.y = 0.f; x2.y.y = 0.f; x2.z.y = 1.f; c0.x.y = 1.f; c0.y.y = 0.f; c0.z.y = 0.f; det.y = 1.f;
    }
    // first step untested (from F it stops only for tets already at a rotation)
    polar_step2(x0, x1, x2, c0, det);
    bool da = !oka, db = !okb;  // done (converged or failed)
#pragma unroll 1
    for (int it = 1; it < 10; ++it) {
        c0 = vcross2(x1, x2);
        det = vdot2(x0, c0);
        if (!da && !(det.x > 0.f)) { oka = false; da = true; }
        if (!db && !(det.y > 0.f)) { okb = false; db = true; }
        if (da && db) return;
        if (da) det.x = 1.f;  // keep the finished lane's arithmetic finite
        if (db) det.y = 1.f;
        const f2 ch = polar_step2(x0, x1, x2, c0, det);
        // step <= 1e-4: the error left after this update is below FP32 resolution
        if (!da && ch.x <= 1e-8f) da = true;
        if (!db && ch.y <= 1e-8f) db = true;
        if (da && db) return;
    }
    if (!da) oka = false;
    if (!db) okb = false;
}

// R = U V^T of the sign-fixed SVD of one tet's F (the rotation closest to F
// among rotations when det F > 0; for inverted tets F - U V^T = U diag(s - 1)
// V^T, so the ARAP-SVD gradient (F - R) / |F - R| is the reference's).
__device__ __forceinline__ void svd_rotation(const M3& F, float R[3][3]) {
    const Svd3 s = svd3(F);
    const float U[3][3] = {{s.u0.x, s.u1.x, s.u2.x}, {s.u0.y, s.u1.y, s.u2.y}, {s.u0.z, s.u1.z, s.u2.z}};
    const float V[3][3] = {{s.v0.x, s.v1.x, s.v2.x}, {s.v0.y, s.v1.y, s.v2.y}, {s.v0.z, s.v1.z, s.v2.z}};
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) R[i][j] = U[i][0] * V[j][0] + U[i][1] * V[j][1] + U[i][2] * V[j][2];
}

__device__ __forceinline__ void acc_tet(const int (&l)[4], const float3 (&d)[4], int nact, float acc_scale,
                                        int32_t* status, int* s_ax, int* s_ay, int* s_az, int* s_cnt) {
    // range check on the sum of the 12 magnitudes (carries NaN/Inf through)
    float dabs = 0.f;
#pragma unroll
    for (int i = 0; i < 4; ++i) dabs += (fabsf(d[i].x) + fabsf(d[i].y)) + fabsf(d[i].z);
    if (!(dabs * acc_scale <= 33554432.f) && status) atomicOr(status, XPBD_STATUS_ACC_RANGE);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        atomicAdd(&s_ax[l[i]], __float2int_rn(d[i].x * acc_scale));
        atomicAdd(&s_ay[l[i]], __float2int_rn(d[i].y * acc_scale));
        atomicAdd(&s_az[l[i]], __float2int_rn(d[i].z * acc_scale));
        atomicAdd(&s_cnt[l[i]], nact);
    }
}

// Projects the tile's tets two per thread per round: tets a = t0 + tid +
// 2 k T and b = a + T (T threads).  Same contract as project_tile_tets for
// the light constraint set (ARAP-SVD and aniso_arap) and, with VOL, the
// volume constraint too; no damping (damped materials read pprev and take
// the one-tet pass).
template <bool VOL>
__device__ __forceinline__ void project_tile_tets_x2(const XpbdParams& prm, const XpbdTiles& T, int tile,
                                                     const float4* s_pos, int* s_ax, int* s_ay, int* s_az,
                                                     int* s_cnt, const float* s_arap_at) {
    const float acc_scale = prm.acc_scale;
    const float arap_skip = arap_skip_threshold(prm.arap_skip_ssq);
    const bool force_svd = (prm.tile_variant & 2) != 0;
    const int t0 = T.tile_tptr[tile], t1 = T.tile_tptr[tile + 1];
    const uint4* tq = reinterpret_cast<const uint4*>(T.tet_q);
    const float4* tb0 = reinterpret_cast<const float4*>(T.tet_b0);
    const float4* tb1 = reinterpret_cast<const float4*>(T.tet_b1);
    const int nthr = int(blockDim.x);
    for (int ta = t0 + int(threadIdx.x); ta < t1; ta += 2 * nthr) {
        const bool hb = ta + nthr < t1;
        const int tb = hb ? ta + nthr : ta;
        const uint4 qa = tq[ta], qb = tq[tb];
        const int la[4] = {int(qa.x & 0xffffu), int(qa.x >> 16), int(qa.y & 0xffffu), int(qa.y >> 16)};
        const int lb[4] = {int(qb.x & 0xffffu), int(qb.x >> 16), int(qb.y & 0xffffu), int(qb.y >> 16)};
        const int ma = min(int(qa.z & 0xffu), XPBD_MAX_MATERIALS - 1), mb = min(int(qb.z & 0xffu), XPBD_MAX_MATERIALS - 1);
        const uint32_t fa = prm.materials[ma].flags, fb = prm.materials[mb].flags;
        float4 pa[4], pb[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            pa[i] = s_pos[la[i]];
            pb[i] = s_pos[lb[i]];
        }
        const float4 ba0 = tb0[ta], ba1 = tb1[ta], bb0 = tb0[tb], bb1 = tb1[tb];
        const float ba2 = T.tet_b2[ta], bb2 = T.tet_b2[tb];
        // B rows packed: B[r][c] of tet a in .x, of tet b in .y
        const f2 B00 = pk(ba0.x, bb0.x), B01 = pk(ba0.y, bb0.y), B02 = pk(ba0.z, bb0.z);
        const f2 B10 = pk(ba0.w, bb0.w), B11 = pk(ba1.x, bb1.x), B12 = pk(ba1.y, bb1.y);
        const f2 B20 = pk(ba1.z, bb1.z), B21 = pk(ba1.w, bb1.w), B22 = pk(ba2, bb2);
        // Ds columns d_k = p_k - p_3
        const V2 p3 = {pk(pa[3].x, pb[3].x), pk(pa[3].y, pb[3].y), pk(pa[3].z, pb[3].z)};
        V2 d0 = vsub2({pk(pa[0].x, pb[0].x), pk(pa[0].y, pb[0].y), pk(pa[0].z, pb[0].z)}, p3);
        V2 d1 = vsub2({pk(pa[1].x, pb[1].x), pk(pa[1].y, pb[1].y), pk(pa[1].z, pb[1].z)}, p3);
        V2 d2 = vsub2({pk(pa[2].x, pb[2].x), pk(pa[2].y, pb[2].y), pk(pa[2].z, pb[2].z)}, p3);
        // F = Ds B; column j of F: row i = d0_i B0j + d1_i B1j + d2_i B2j
        auto col = [&](f2 b0j, f2 b1j, f2 b2j) -> V2 {
            return {fma2(d2.x, b2j, fma2(d1.x, b1j, mul2(d0.x, b0j))), fma2(d2.y, b2j, fma2(d1.y, b1j, mul2(d0.y, b0j))),
                    fma2(d2.z, b2j, fma2(d1.z, b1j, mul2(d0.z, b0j)))};
        };
        const V2 F0 = col(B00, B10, B20), F1 = col(B01, B11, B21), F2 = col(B02, B12, B22);
        const f2 w0 = pk(pa[0].w, pb[0].w), w1 = pk(pa[1].w, pb[1].w), w2 = pk(pa[2].w, pb[2].w),
                 w3 = pk(pa[3].w, pb[3].w);
        float3 da[4], db[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            da[i] = make_float3(0.f, 0.f, 0.f);
            db[i] = make_float3(0.f, 0.f, 0.f);
        }
        int na = 0, nb = 0;
        const bool arap_a = (fa & XPBD_MAT_ARAPSVD) != 0, arap_b = hb && (fb & XPBD_MAT_ARAPSVD) != 0;
        if (arap_a || arap_b) {
            V2 r0 = F0, r1 = F1, r2 = F2;
            bool oka = false, okb = false;
            if (!force_svd) polar_rotation2(r0, r1, r2, oka, okb);
            if (!oka || !okb) {
                // SVD fallback per tet (inverted or degenerate): R = U V^T
#pragma unroll
                for (int lane = 0; lane < 2; ++lane) {
                    if (lane == 0 ? oka : okb) continue;
                    M3 F;
                    F.m[0][0] = lane ? F0.x.y : F0.x.x; F.m[1][0] = lane ? F0.y.y : F0.y.x; F.m[2][0] = lane ? F0.z.y : F0.z.x;
                    F.m[0][1] = lane ? F1.x.y : F1.x.x; F.m[1][1] = lane ? F1.y.y : F1.y.x; F.m[2][1] = lane ? F1.z.y : F1.z.x;
                    F.m[0][2] = lane ? F2.x.y : F2.x.x; F.m[1][2] = lane ? F2.y.y : F2.y.x; F.m[2][2] = lane ? F2.z.y : F2.z.x;
                    float R[3][3];
                    svd_rotation(F, R);
                    if (lane == 0) {
                        r0.x.x = R[0][0]; r0.y.x = R[1][0]; r0.z.x = R[2][0];
                        r1.x.x = R[0][1]; r1.y.x = R[1][1]; r1.z.x = R[2][1];
                        r2.x.x = R[0][2]; r2.y.x = R[1][2]; r2.z.x = R[2][2];
                    } else {
                        r0.x.y = R[0][0]; r0.y.y = R[1][0]; r0.z.y = R[2][0];
                        r1.x.y = R[0][1]; r1.y.y = R[1][1]; r1.z.y = R[2][1];
                        r2.x.y = R[0][2]; r2.y.y = R[1][2]; r2.z.y = R[2][2];
                    }
                }
            }
            // G = F - R (columns), ssq = |G|_F^2 in row-major order
            V2 g0 = vsub2(F0, r0), g1 = vsub2(F1, r1), g2 = vsub2(F2, r2);
            f2 ssq = mul2(g0.x, g0.x);
            ssq = fma2(g1.x, g1.x, ssq);
            ssq = fma2(g2.x, g2.x, ssq);
            ssq = fma2(g0.y, g0.y, ssq);
            ssq = fma2(g1.y, g1.y, ssq);
            ssq = fma2(g2.y, g2.y, ssq);
            ssq = fma2(g0.z, g0.z, ssq);
            ssq = fma2(g1.z, g1.z, ssq);
            ssq = fma2(g2.z, g2.z, ssq);
            bool acta = arap_a && !(ssq.x < arap_skip), actb = arap_b && !(ssq.y < arap_skip);
            if (acta || actb) {
                const f2 invC = pk(rsqrtf(ssq.x), rsqrtf(ssq.y));
                const f2 C = mul2(ssq, invC);
                g0 = {mul2(g0.x, invC), mul2(g0.y, invC), mul2(g0.z, invC)};
                g1 = {mul2(g1.x, invC), mul2(g1.y, invC), mul2(g1.z, invC)};
                g2 = {mul2(g2.x, invC), mul2(g2.y, invC), mul2(g2.z, invC)};
                // gradient rows: grad_k[a] = sum_j G[a][j] B[k][j], G's columns g0..g2
                auto row = [&](f2 bk0, f2 bk1, f2 bk2) -> V2 {
                    return {fma2(g2.x, bk2, fma2(g1.x, bk1, mul2(g0.x, bk0))),
                            fma2(g2.y, bk2, fma2(g1.y, bk1, mul2(g0.y, bk0))),
                            fma2(g2.z, bk2, fma2(g1.z, bk1, mul2(g0.z, bk0)))};
                };
                const V2 q0 = row(B00, B01, B02), q1 = row(B10, B11, B12), q2 = row(B20, B21, B22);
                const V2 s01 = {add2(q0.x, q1.x), add2(q0.y, q1.y), add2(q0.z, q1.z)};
                const V2 q3 = {neg2(add2(s01.x, q2.x)), neg2(add2(s01.y, q2.y)), neg2(add2(s01.z, q2.z))};
                f2 wsum = mul2(w0, vdot2(q0, q0));
                wsum = fma2(w1, vdot2(q1, q1), wsum);
                wsum = fma2(w2, vdot2(q2, q2), wsum);
                wsum = fma2(w3, vdot2(q3, q3), wsum);
                acta = acta && wsum.x != 0.f;
                actb = actb && wsum.y != 0.f;
                const f2 den = add2(wsum, pk(s_arap_at[ma], s_arap_at[mb]));
                const f2 dL = pk(-__fdividef(C.x, den.x), -__fdividef(C.y, den.y));
                const f2 s0 = mul2(dL, w0), s1 = mul2(dL, w1), s2 = mul2(dL, w2), s3 = mul2(dL, w3);
                const V2 e0 = {mul2(s0, q0.x), mul2(s0, q0.y), mul2(s0, q0.z)};
                const V2 e1 = {mul2(s1, q1.x), mul2(s1, q1.y), mul2(s1, q1.z)};
                const V2 e2 = {mul2(s2, q2.x), mul2(s2, q2.y), mul2(s2, q2.z)};
                const V2 e3 = {mul2(s3, q3.x), mul2(s3, q3.y), mul2(s3, q3.z)};
                if (acta) {
                    da[0] = make_float3(e0.x.x, e0.y.x, e0.z.x);
                    da[1] = make_float3(e1.x.x, e1.y.x, e1.z.x);
                    da[2] = make_float3(e2.x.x, e2.y.x, e2.z.x);
                    da[3] = make_float3(e3.x.x, e3.y.x, e3.z.x);
                    na = 1;
                }
                if (actb) {
                    db[0] = make_float3(e0.x.y, e0.y.y, e0.z.y);
                    db[1] = make_float3(e1.x.y, e1.y.y, e1.z.y);
                    db[2] = make_float3(e2.x.y, e2.y.y, e2.z.y);
                    db[3] = make_float3(e3.x.y, e3.y.y, e3.z.y);
                    nb = 1;
                }
            }
        }
        // volume (tet_volume_update_xpbd_fn, solve_kernels.py:187-281, undamped):
        // gradients are the face cross products / 6 (pt3 reference), C = V - V0
        if constexpr (VOL) {
            const bool vola = (fa & XPBD_MAT_VOLUME) != 0, volb = hb && (fb & XPBD_MAT_VOLUME) != 0;
            if (vola || volb) {
                const f2 sixth = pk(1.f / 6.f, 1.f / 6.f);
                const V2 c0 = vcross2(d1, d2), c1 = vcross2(d2, d0), c2 = vcross2(d0, d1);
                const f2 vol = mul2(vdot2(c2, d2), sixth);
                const V2 v0 = {mul2(c0.x, sixth), mul2(c0.y, sixth), mul2(c0.z, sixth)};
                const V2 v1 = {mul2(c1.x, sixth), mul2(c1.y, sixth), mul2(c1.z, sixth)};
                const V2 v2 = {mul2(c2.x, sixth), mul2(c2.y, sixth), mul2(c2.z, sixth)};
                const V2 s01 = {add2(v0.x, v1.x), add2(v0.y, v1.y), add2(v0.z, v1.z)};
                const V2 v3 = {neg2(add2(s01.x, v2.x)), neg2(add2(s01.y, v2.y)), neg2(add2(s01.z, v2.z))};
                f2 ws = mul2(w0, vdot2(v0, v0));
                ws = fma2(w1, vdot2(v1, v1), ws);
                ws = fma2(w2, vdot2(v2, v2), ws);
                ws = fma2(w3, vdot2(v3, v3), ws);
                const bool oka = vola && ws.x > 1e-9f, okb = volb && ws.y > 1e-9f;
                if (oka || okb) {
                    const float dt2 = prm.dt * prm.dt;
                    const f2 alpha = pk((1.f / prm.materials[ma].vol_k) / dt2, (1.f / prm.materials[mb].vol_k) / dt2);
                    const f2 C = sub2(vol, pk(__uint_as_float(qa.w), __uint_as_float(qb.w)));
                    const f2 den = add2(ws, alpha);
                    const f2 dl = pk(-C.x / den.x, -C.y / den.y);
                    const f2 s0 = mul2(dl, w0), s1 = mul2(dl, w1), s2 = mul2(dl, w2), s3 = mul2(dl, w3);
                    const V2 e0 = {mul2(s0, v0.x), mul2(s0, v0.y), mul2(s0, v0.z)};
                    const V2 e1 = {mul2(s1, v1.x), mul2(s1, v1.y), mul2(s1, v1.z)};
                    const V2 e2 = {mul2(s2, v2.x), mul2(s2, v2.y), mul2(s2, v2.z)};
                    const V2 e3 = {mul2(s3, v3.x), mul2(s3, v3.y), mul2(s3, v3.z)};
                    if (oka) {
                        da[0] = da[0] + make_float3(e0.x.x, e0.y.x, e0.z.x);
                        da[1] = da[1] + make_float3(e1.x.x, e1.y.x, e1.z.x);
                        da[2] = da[2] + make_float3(e2.x.x, e2.y.x, e2.z.x);
                        da[3] = da[3] + make_float3(e3.x.x, e3.y.x, e3.z.x);
                        na += 1;
                    }
                    if (okb) {
                        db[0] = db[0] + make_float3(e0.x.y, e0.y.y, e0.z.y);
                        db[1] = db[1] + make_float3(e1.x.y, e1.y.y, e1.z.y);
                        db[2] = db[2] + make_float3(e2.x.y, e2.y.y, e2.z.y);
                        db[3] = db[3] + make_float3(e3.x.y, e3.y.y, e3.z.y);
                        nb += 1;
                    }
                }
            }
        }
        // aniso_arap (one muscle), per tet, added to the ARAP term (the scalar
        // pass sums the two in the other order: at most one rounding apart)
        auto aniso = [&](const float4 (&pp)[4], int t, int m, int lane, float3 (&dd)[4], int& n) {
            M3 F, B;
            F.m[0][0] = lane ? F0.x.y : F0.x.x; F.m[1][0] = lane ? F0.y.y : F0.y.x; F.m[2][0] = lane ? F0.z.y : F0.z.x;
            F.m[0][1] = lane ? F1.x.y : F1.x.x; F.m[1][1] = lane ? F1.y.y : F1.y.x; F.m[2][1] = lane ? F1.z.y : F1.z.x;
            F.m[0][2] = lane ? F2.x.y : F2.x.x; F.m[1][2] = lane ? F2.y.y : F2.y.x; F.m[2][2] = lane ? F2.z.y : F2.z.x;
            B.m[0][0] = lane ? B00.y : B00.x; B.m[0][1] = lane ? B01.y : B01.x; B.m[0][2] = lane ? B02.y : B02.x;
            B.m[1][0] = lane ? B10.y : B10.x; B.m[1][1] = lane ? B11.y : B11.x; B.m[1][2] = lane ? B12.y : B12.x;
            B.m[2][0] = lane ? B20.y : B20.x; B.m[2][1] = lane ? B21.y : B21.x; B.m[2][2] = lane ? B22.y : B22.x;
            const float4 fbv = reinterpret_cast<const float4*>(T.tet_fiber)[t];
            if (con_aniso(pp, B, F, f3(fbv), fbv.w, T.tet_act[t], prm.materials[m].aniso_k, prm.contraction_ratio,
                          prm.fiber_stiffness_scale, prm.dt, 1.f, dd))
                n += 1;
        };
        if (fa & XPBD_MAT_ANISO) aniso(pa, ta, ma, 0, da, na);
        if (hb && (fb & XPBD_MAT_ANISO)) aniso(pb, tb, mb, 1, db, nb);
        if (na) acc_tet(la, da, na, acc_scale, prm.status, s_ax, s_ay, s_az, s_cnt);
        if (nb) acc_tet(lb, db, nb, acc_scale, prm.status, s_ax, s_ay, s_az, s_cnt);
    }
}

}  // namespace xpbd
