// Device math and per-constraint XPBD projections for sm_100a.
//
// Each constraint function restates one reference Warp kernel
// (chunleili/rlmuscleV2 src/muscle/constraint/solve_kernels.py) for the
// Jacobi path (use_jacobi=1, Lagrange multipliers zeroed every iteration so
// L == 0), returning the per-vertex position deltas that the reference
// passes to update_dP (solve_kernels.py:52-56).  Positions arrive as float4
// with the inverse mass in .w (get_inv_mass_fn, solve_kernels.py:71-80, is
// folded into that lane at upload time).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace xpbd {

struct M3 { float m[3][3]; };

__device__ __forceinline__ float3 f3(float4 a) { return make_float3(a.x, a.y, a.z); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator-(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float3 operator*(float s, float3 a) { return make_float3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float3 operator/(float3 a, float s) { return make_float3(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross(float3 a, float3 b) {
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float len(float3 a) { return sqrtf(dot(a, a)); }

// F = Ds * B with Ds columns (c0, c1, c2) -- engine.py / solve_kernels.py layout.
__device__ __forceinline__ M3 deformation(float3 c0, float3 c1, float3 c2, const M3& B) {
    const float d[3][3] = {{c0.x, c1.x, c2.x}, {c0.y, c1.y, c2.y}, {c0.z, c1.z, c2.z}};
    M3 F;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) F.m[i][j] = d[i][0] * B.m[0][j] + d[i][1] * B.m[1][j] + d[i][2] * B.m[2][j];
    return F;
}

__device__ __forceinline__ float det3(const M3& M) {
    return M.m[0][0] * (M.m[1][1] * M.m[2][2] - M.m[1][2] * M.m[2][1])
         - M.m[0][1] * (M.m[1][0] * M.m[2][2] - M.m[1][2] * M.m[2][0])
         + M.m[0][2] * (M.m[1][0] * M.m[2][1] - M.m[1][1] * M.m[2][0]);
}

// grad_k[a] = sum_j G[a][j] * B[k][j]   (solve_kernels.py:1276-1288)
__device__ __forceinline__ float3 grad_row(const M3& G, const M3& B, int k) {
    return make_float3(G.m[0][0] * B.m[k][0] + G.m[0][1] * B.m[k][1] + G.m[0][2] * B.m[k][2],
                       G.m[1][0] * B.m[k][0] + G.m[1][1] * B.m[k][1] + G.m[1][2] * B.m[k][2],
                       G.m[2][0] * B.m[k][0] + G.m[2][1] * B.m[k][1] + G.m[2][2] * B.m[k][2]);
}

// ---------------------------------------------------------------------------
// Sign-fixed 3x3 SVD: F = U diag(s) V^T with U, V rotations, s0 >= s1 >= |s2|,
// sign(s2) = sign(det F) -- the factorisation ssvd_fn (solve_kernels.py:85-112)
// produces.  Method: cyclic Jacobi eigen-decomposition of the symmetric
// S = F^T F (Jacobi rotations with the Rutishauser update formulas, Golub &
// Van Loan sec. 8.5), eigenvalues sorted descending, then U is built from
// F V: u0 = F v0/|F v0|, u1 by Gram-Schmidt, u2 = u0 x u1, so U is a rotation
// by construction and s2 = u2 . (F v2) carries the sign of det F.  Singular
// values are read off |F v_k| (second-order accurate in the eigenvector
// error), not sqrt of the eigenvalues.
struct Svd3 {
    float3 u0, u1, u2;  // columns of U
    float3 v0, v1, v2;  // columns of V
    float s0, s1, s2;
};

__device__ __forceinline__ void jacobi_rot(float& spp, float& sqq, float& spq, float& srp, float& srq,
                                           float3& vp, float3& vq) {
    // tan of the rotation angle, t = sign(theta)/(|theta| + sqrt(theta^2 + 1)) with
    // theta = (sqq - spp)/(2 spq), written without dividing by spq:
    // t = spq / (h + sign(h) sqrt(h^2 + spq^2)), h = (sqq - spp)/2.  Branch-free;
    // t = 0 when spq = 0 and h = 0.
    const float h = 0.5f * (sqq - spp);
    const float r = sqrtf(fmaf(h, h, spq * spq));
    const float den = h + copysignf(r, h);
    const float t = den != 0.f ? __fdividef(spq, den) : 0.f;
    const float c = rsqrtf(fmaf(t, t, 1.f));
    const float s = t * c;
    spp = fmaf(-t, spq, spp);
    sqq = fmaf(t, spq, sqq);
    spq = 0.f;
    const float rp = srp, rq = srq;
    srp = c * rp - s * rq;
    srq = s * rp + c * rq;
    const float3 a = vp, b = vq;
    vp = make_float3(c * a.x - s * b.x, c * a.y - s * b.y, c * a.z - s * b.z);
    vq = make_float3(s * a.x + c * b.x, s * a.y + c * b.y, s * a.z + c * b.z);
}

__device__ __forceinline__ void swap3(float3& a, float3& b) { float3 t = a; a = b; b = t; }

__device__ __forceinline__ Svd3 svd3(const M3& F) {
    // S = F^T F (upper triangle)
    float s00 = F.m[0][0] * F.m[0][0] + F.m[1][0] * F.m[1][0] + F.m[2][0] * F.m[2][0];
    float s01 = F.m[0][0] * F.m[0][1] + F.m[1][0] * F.m[1][1] + F.m[2][0] * F.m[2][1];
    float s02 = F.m[0][0] * F.m[0][2] + F.m[1][0] * F.m[1][2] + F.m[2][0] * F.m[2][2];
    float s11 = F.m[0][1] * F.m[0][1] + F.m[1][1] * F.m[1][1] + F.m[2][1] * F.m[2][1];
    float s12 = F.m[0][1] * F.m[0][2] + F.m[1][1] * F.m[1][2] + F.m[2][1] * F.m[2][2];
    float s22 = F.m[0][2] * F.m[0][2] + F.m[1][2] * F.m[1][2] + F.m[2][2] * F.m[2][2];
    Svd3 r;
    r.v0 = make_float3(1.f, 0.f, 0.f);
    r.v1 = make_float3(0.f, 1.f, 0.f);
    r.v2 = make_float3(0.f, 0.f, 1.f);
#pragma unroll 1
    for (int sweep = 0; sweep < 4; ++sweep) {
        // converged when the off-diagonal mass is at FP32 rounding level
        const float off = s01 * s01 + s02 * s02 + s12 * s12;
        const float dia = s00 * s00 + s11 * s11 + s22 * s22;
        if (off <= 1e-13f * dia) break;
        // plane (0,1), third index 2: s20=s02, s21=s12
        jacobi_rot(s00, s11, s01, s02, s12, r.v0, r.v1);
        // plane (0,2), third index 1: s10=s01, s12
        jacobi_rot(s00, s22, s02, s01, s12, r.v0, r.v2);
        // plane (1,2), third index 0: s01, s02
        jacobi_rot(s11, s22, s12, s01, s02, r.v1, r.v2);
    }
    // sort eigenvalues descending (columns of V follow)
    float l0 = s00, l1 = s11, l2 = s22, tl;
    if (l1 > l0) { tl = l0; l0 = l1; l1 = tl; swap3(r.v0, r.v1); }
    if (l2 > l0) { tl = l0; l0 = l2; l2 = tl; swap3(r.v0, r.v2); }
    if (l2 > l1) { tl = l1; l1 = l2; l2 = tl; swap3(r.v1, r.v2); }
    if (dot(r.v0, cross(r.v1, r.v2)) < 0.f) r.v2 = -r.v2;
    auto Fv = [&](float3 v) {
        return make_float3(F.m[0][0] * v.x + F.m[0][1] * v.y + F.m[0][2] * v.z,
                           F.m[1][0] * v.x + F.m[1][1] * v.y + F.m[1][2] * v.z,
                           F.m[2][0] * v.x + F.m[2][1] * v.y + F.m[2][2] * v.z);
    };
    const float3 b0 = Fv(r.v0), b1 = Fv(r.v1), b2 = Fv(r.v2);
    const float n0 = len(b0);
    r.u0 = n0 > 1e-30f ? rsqrtf(dot(b0, b0)) * b0 : make_float3(1.f, 0.f, 0.f);
    r.s0 = n0;
    const float pr = dot(r.u0, b1);
    const float3 w = b1 - pr * r.u0;
    const float n1 = len(w);
    if (n1 > 1e-30f * fmaxf(n0, 1.f)) {
        r.u1 = rsqrtf(dot(w, w)) * w;
    } else {
        const float a0 = fabsf(r.u0.x), a1 = fabsf(r.u0.y), a2 = fabsf(r.u0.z);
        float3 e = (a0 <= a1 && a0 <= a2) ? make_float3(1.f, 0.f, 0.f)
                   : (a1 <= a2 ? make_float3(0.f, 1.f, 0.f) : make_float3(0.f, 0.f, 1.f));
        float3 c = cross(r.u0, e);
        r.u1 = c / len(c);
    }
    r.s1 = dot(r.u1, b1);
    r.u2 = cross(r.u0, r.u1);
    r.s2 = dot(r.u2, b2);
    return r;
}

// ---------------------------------------------------------------------------
// Material table entry (constraints a tet carries and their parameters).
enum : uint32_t {
    MAT_ARAPSVD = 1u << 0,
    MAT_VOLUME = 1u << 1,
    MAT_ANISO = 1u << 2,
    MAT_SNH = 1u << 3,
    MAT_DAMPED = 1u << 4,  // some constraint of this material reads pprev
};

// Rotation factor R of F = R S for det F > 0, by Higham's scaled Newton
// iteration X <- (g X + (g X)^-T) / 2, g = det(X)^(-1/3) (N. J. Higham,
// "Computing the polar decomposition with applications", SIAM J. Sci. Stat.
// Comput. 7, 1986).  With the cofactor matrix C = det(X) X^-T (columns: cross
// products of X's columns) the step is X <- (g/2) (X + g C).  The iteration is
// invariant to a positive factor on X (g X does not change), so the factor
// g/2 is dropped and X <- X + g C is iterated (one FMA per entry); only the
// last step is taken in the scaled form.  The iteration keeps det X > 0 when it
// starts there, so after the start test the first two steps run untested:
// nearly every tet needs two or three, a warp runs as many as its slowest
// lane, and a converged tet stays put under a further step.  From the third
// step on, the step of the unit-determinant iterates, (g/2)(g C - X), is
// tested.  Returns false (caller falls back to the SVD) for det F <= tiny or
// when 10 steps do not converge.
// The start test of polar_rotation: F's columns, the first cofactor column,
// det F, and whether det F > 1e-6 |F|_F^3 (squared to avoid the square
// root).  Tets that fail it take the SVD.
__device__ __forceinline__ bool polar_start(const M3& F, float3& x0, float3& x1, float3& x2, float3& c0, float& det) {
    x0 = make_float3(F.m[0][0], F.m[1][0], F.m[2][0]);
    x1 = make_float3(F.m[0][1], F.m[1][1], F.m[2][1]);
    x2 = make_float3(F.m[0][2], F.m[1][2], F.m[2][2]);
    const float n2 = dot(x0, x0) + dot(x1, x1) + dot(x2, x2);
    c0 = cross(x1, x2);
    det = dot(x0, c0);
    return det > 0.f && det * det > 1e-12f * (n2 * n2 * n2);
}

__device__ __forceinline__ bool polar_start_ok(const M3& F) {
    float3 x0, x1, x2, c0;
    float det;
    return polar_start(F, x0, x1, x2, c0, det);
}

__device__ __forceinline__ bool polar_rotation(const M3& F, M3& R) {
    float3 x0, x1, x2, c0;
    float det;
    if (!polar_start(F, x0, x1, x2, c0, det)) return false;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const float3 c1 = cross(x2, x0), c2 = cross(x0, x1);
        const float g = __powf(det, -0.33333334f);
        x0 = x0 + g * c0;
        x1 = x1 + g * c1;
        x2 = x2 + g * c2;
        c0 = cross(x1, x2);
        det = dot(x0, c0);
    }
#pragma unroll 1
    for (int it = 2; it < 10; ++it) {
        if (!(det > 0.f)) return false;
        const float3 c1 = cross(x2, x0), c2 = cross(x0, x1);
        const float g = __powf(det, -0.33333334f);
        const float3 d0 = g * c0 - x0, d1 = g * c1 - x1, d2 = g * c2 - x2;
        const float dd = dot(d0, d0) + dot(d1, d1) + dot(d2, d2);
        // step <= 1e-4: Newton's quadratic convergence leaves an error ~|step|^2/2 = 5e-9
        // after this update, below the FP32 resolution of R's entries.  The last step
        // is taken in the scaled form (g X + C / (g det)) / 2, whose fixed point does
        // not depend on the error of the fast power g (it enters at second order).
        if (dd * (g * g) <= 4e-8f) {
            const float a = 0.5f * g, h = __fdividef(0.5f, g * det);
            const float3 r0 = a * x0 + h * c0, r1 = a * x1 + h * c1, r2 = a * x2 + h * c2;
            R.m[0][0] = r0.x; R.m[1][0] = r0.y; R.m[2][0] = r0.z;
            R.m[0][1] = r1.x; R.m[1][1] = r1.y; R.m[2][1] = r1.z;
            R.m[0][2] = r2.x; R.m[1][2] = r2.y; R.m[2][2] = r2.z;
            return true;
        }
        x0 = (x0 + x0) + d0;  // X + g C
        x1 = (x1 + x1) + d1;
        x2 = (x2 + x2) + d2;
        c0 = cross(x1, x2);
        det = dot(x0, c0);
    }
    return false;
}

// solve_tetarap_svd_kernel, solve_kernels.py:1194-1307 (Jacobi branch).
// With the sign-fixed SVD F = U diag(s) V^T (U, V rotations) the constraint is
// C = ||s - 1|| = ||F - U V^T||_F and dC/dF = U diag((s-1)/C) V^T = (F - U V^T)/C,
// U V^T being the rotation nearest F.  For det F > 0 that rotation is the polar
// factor, obtained without the SVD; inverted or degenerate tets use the SVD.
// at = alpha / dt^2 with alpha = 1 / stiffness, evaluated once per material
// per launch (arap_alpha_tilde) in the reference's operation order.
__device__ __forceinline__ float arap_alpha_tilde(float k, float dt) {
    const float alpha = 1.f / k;
    return alpha / (dt * dt);
}

__device__ __forceinline__ float arap_skip_threshold(float v) {
    return v == 0.f ? 1.0e-12f : (v < 0.f ? 1.0e-38f : v);
}

// The per-vertex delta is added as (dL w_i scale) grad_i with grad built from
// the unnormalised G = F - R and 1/C folded into that scale factor (the scale
// is the caller's fixed-point factor, a power of two, so it changes no
// rounding); acc receives the scaled deltas.
__device__ __forceinline__ bool con_arapsvd(const float4 p[4], const M3& B, const M3& F, float at, float skip_ssq,
                                            float scale, float3 (&acc)[4], bool force_svd = false) {
    M3 G;
    M3 R;
    float ssq;
    if (!force_svd && polar_rotation(F, R)) {
        ssq = 0.f;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                G.m[i][j] = F.m[i][j] - R.m[i][j];
                ssq += G.m[i][j] * G.m[i][j];
            }
        if (ssq < skip_ssq) return false;
    } else {
        // F - U V^T = U diag(s - 1) V^T
        const Svd3 s = svd3(F);
        const float a = s.s0 - 1.f, b = s.s1 - 1.f, c = s.s2 - 1.f;
        ssq = a * a + b * b + c * c;
        if (ssq < skip_ssq) return false;
        const float U[3][3] = {{s.u0.x, s.u1.x, s.u2.x}, {s.u0.y, s.u1.y, s.u2.y}, {s.u0.z, s.u1.z, s.u2.z}};
        const float V[3][3] = {{s.v0.x, s.v1.x, s.v2.x}, {s.v0.y, s.v1.y, s.v2.y}, {s.v0.z, s.v1.z, s.v2.z}};
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) G.m[i][j] = U[i][0] * V[j][0] * a + U[i][1] * V[j][1] * b + U[i][2] * V[j][2] * c;
    }
    const float invC = rsqrtf(ssq);
    const float C = ssq * invC;
    // raw gradient rows (F - R) B^T; the constraint gradient is invC times them
    float3 g[4];
    g[0] = grad_row(G, B, 0);
    g[1] = grad_row(G, B, 1);
    g[2] = grad_row(G, B, 2);
    g[3] = (-g[0] - g[1]) - g[2];
    const float wraw = p[0].w * dot(g[0], g[0]) + p[1].w * dot(g[1], g[1]) + p[2].w * dot(g[2], g[2]) + p[3].w * dot(g[3], g[3]);
    if (wraw == 0.f) return false;
    const float dL = -C / (wraw * (invC * invC) + at);
    const float k = dL * invC * scale;
#pragma unroll
    for (int i = 0; i < 4; ++i) acc[i] = acc[i] + (k * p[i].w) * g[i];
    return true;
}

// solve_tetvolume_kernel + tet_volume_update_xpbd_fn, solve_kernels.py:553-585, 187-281.
__device__ __forceinline__ bool con_volume(const float4 p[4], const float4* q, float V0, float k, float kd, float dt,
                                           float scale, float3 (&acc)[4]) {
    const float3 p3 = f3(p[3]);
    const float3 d0 = f3(p[0]) - p3, d1 = f3(p[1]) - p3, d2 = f3(p[2]) - p3;
    float3 g[4];
    g[0] = cross(d1, d2) / 6.f;
    g[1] = cross(d2, d0) / 6.f;
    g[2] = cross(d0, d1) / 6.f;
    g[3] = -((g[0] + g[1]) + g[2]);
    const float ws = p[0].w * dot(g[0], g[0]) + p[1].w * dot(g[1], g[1]) + p[2].w * dot(g[2], g[2]) + p[3].w * dot(g[3], g[3]);
    if (!(ws > 1e-9f)) return false;
    const float volume = dot(cross(d0, d1), d2) / 6.f;
    float alpha = 1.f / k;
    alpha = alpha / (dt * dt);
    const float C = volume - V0;
    float dsum = 0.f, gamma = 1.f;
    if (kd > 0.f) {
        const float beta = k * kd * dt * dt;
        gamma = alpha * beta / dt;
        dsum = dot(g[0], f3(p[0]) - f3(q[0])) + dot(g[1], f3(p[1]) - f3(q[1])) + dot(g[2], f3(p[2]) - f3(q[2])) +
               dot(g[3], f3(p[3]) - f3(q[3]));
        dsum = dsum * gamma;
        gamma = gamma + 1.f;
    }
    const float dl = (-C - dsum) / (gamma * ws + alpha) * scale;
#pragma unroll
    for (int i = 0; i < 4; ++i) acc[i] = acc[i] + (dl * p[i].w) * g[i];
    return true;
}

// solve_tet_aniso_arap_kernel, solve_kernels.py:1310-1426.  f0 is the
// normalised mean fiber direction of the tet's 4 vertices (static, built at
// upload); a zero f0 marks a tet whose mean fiber vanished (fn < 1e-9).
__device__ __forceinline__ bool con_aniso(const float4 p[4], const M3& B, const M3& F, float3 f0, float tendon,
                                          float act, float k, float ratio, float kscale, float dt, float scale,
                                          float3 (&acc)[4]) {
    const float3 d = make_float3(F.m[0][0] * f0.x + F.m[0][1] * f0.y + F.m[0][2] * f0.z,
                                 F.m[1][0] * f0.x + F.m[1][1] * f0.y + F.m[1][2] * f0.z,
                                 F.m[2][0] * f0.x + F.m[2][1] * f0.y + F.m[2][2] * f0.z);
    const float s = len(d);
    if (s < 1.0e-9f) return false;
    const float detF = det3(F);
    if (detF <= 0.f || s > 1.5f) return false;
    const float belly = 1.f - tendon;
    const float fiberscale = 1.f - belly * act * ratio;
    const float diff = s - fiberscale;
    const float C = 0.5f * diff * diff;
    const float gs = diff / s;
    const float dd[3] = {d.x, d.y, d.z}, ff[3] = {f0.x, f0.y, f0.z};
    M3 G;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) G.m[i][j] = gs * (dd[i] * ff[j]);
    float3 g[4];
    g[0] = grad_row(G, B, 0);
    g[1] = grad_row(G, B, 1);
    g[2] = grad_row(G, B, 2);
    g[3] = (-g[0] - g[1]) - g[2];
    const float wsum = p[0].w * dot(g[0], g[0]) + p[1].w * dot(g[1], g[1]) + p[2].w * dot(g[2], g[2]) + p[3].w * dot(g[3], g[3]);
    if (wsum < 1.0e-20f) return false;
    const float sv = k * kscale;
    const float at = (1.f / sv) / (dt * dt);
    const float dL = -C / (wsum + at) * scale;
#pragma unroll
    for (int i = 0; i < 4; ++i) acc[i] = acc[i] + (dL * p[i].w) * g[i];
    return true;
}

// solve_tetsnh_kernel + tet_snh_update_xpbd_fn, solve_kernels.py:1587-1617, 1429-1584.
__device__ __forceinline__ bool con_snh(const float4 p[4], const float4* q, const M3& B, const M3& F, float V0,
                                        float mu, float lam, float kd, float dt, float scale, float3 (&acc)[4]) {
    float Ic = 0.f;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) Ic += F.m[i][j] * F.m[i][j];
    const float rs = sqrtf(fmaxf(Ic, 1.0e-12f));
    const float dC = rs - 1.7320508075688772f;
    if (rs < 1.0e-6f) return false;
    const float inv_rs = 1.f / rs;
    M3 Fn;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) Fn.m[i][j] = F.m[i][j] * inv_rs;
    float3 dg[4], hg[4];
#pragma unroll
    for (int k = 0; k < 3; ++k)
        dg[k] = make_float3(B.m[k][0] * Fn.m[0][0] + B.m[k][1] * Fn.m[0][1] + B.m[k][2] * Fn.m[0][2],
                            B.m[k][0] * Fn.m[1][0] + B.m[k][1] * Fn.m[1][1] + B.m[k][2] * Fn.m[1][2],
                            B.m[k][0] * Fn.m[2][0] + B.m[k][1] * Fn.m[2][1] + B.m[k][2] * Fn.m[2][2]);
    dg[3] = (-dg[0] - dg[1]) - dg[2];
    float dsw = 0.f;
#pragma unroll
    for (int i = 0; i < 4; ++i) dsw += p[i].w * dot(dg[i], dg[i]);
    if (dsw == 0.f) return false;
    const float asnh = 1.f + mu / lam;
    const float hC = det3(F) - asnh;
    const float3 p3 = f3(p[3]);
    const float3 c0 = f3(p[0]) - p3, c1 = f3(p[1]) - p3, c2 = f3(p[2]) - p3;
    const float av = fmaxf(fabsf(V0), 1.0e-20f);
    const float inv_detDm = 1.f / fmaxf(fabsf(V0) * 6.f, 1.0e-20f);
    hg[0] = inv_detDm * cross(c1, c2);
    hg[1] = inv_detDm * cross(c2, c0);
    hg[2] = inv_detDm * cross(c0, c1);
    hg[3] = (-hg[0] - hg[1]) - hg[2];
    float hsw = 0.f, dh = 0.f;
#pragma unroll
    for (int i = 0; i < 4; ++i) hsw += p[i].w * dot(hg[i], hg[i]);
    if (hsw == 0.f) return false;
#pragma unroll
    for (int i = 0; i < 4; ++i) dh += p[i].w * dot(dg[i], hg[i]);
    const float dalpha = 1.f / (mu * av * dt * dt);
    const float halpha = 1.f / (lam * av * dt * dt);
    float ddamp = 0.f, dgam = 1.f, hdamp = 0.f, hgam = 1.f;
    if (kd > 0.f) {
        const float dbeta = mu * av * kd * dt * dt, hbeta = lam * av * kd * dt * dt;
        dgam = dalpha * dbeta / dt;
        hgam = halpha * hbeta / dt;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const float3 dv = f3(p[i]) - f3(q[i]);
            ddamp += dot(dg[i], dv);
            hdamp += dot(hg[i], dv);
        }
        ddamp = ddamp * dgam;
        hdamp = hdamp * hgam;
        dgam = dgam + 1.f;
        hgam = hgam + 1.f;
    }
    const float Axx = dgam * dsw + dalpha, Ayy = hgam * hsw + halpha;
    const float detA = Axx * Ayy - dh * dh;
    if (detA < 1.0e-8f) return false;
    const float invd = 1.f / detA;
    const float db = -dC - ddamp;
    const float hb = -hC - hdamp;
    const float ddL = invd * (Ayy * db - dh * hb) * scale;
    const float hdL = invd * (Axx * hb - dh * db) * scale;
#pragma unroll
    for (int i = 0; i < 4; ++i) acc[i] = acc[i] + p[i].w * (ddL * dg[i] + hdL * hg[i]);
    return true;
}

// attach_bilateral_update_fn (Jacobi branch), solve_kernels.py:462-526, for
// restlength-parameterised point attachment to a target.  Returns the delta
// for the attached vertex.
__device__ __forceinline__ bool con_attach(float4 p, float3 prev, float3 tgt, float restlength, float k, float kd,
                                           float dt, float3& out) {
    const float im = p.w;
    if (im == 0.f) return false;
    float3 n = f3(p) - tgt;
    const float d = len(n);
    if (!(d >= 1.0e-6f)) return false;
    float alpha = 1.f / k;
    alpha = alpha / (dt * dt);
    const float C = d - restlength;
    n = n / d;
    float dsum = 0.f, gamma = 1.f;
    if (kd > 0.f) {
        const float beta = k * kd * dt * dt;
        gamma = alpha * beta / dt;
        dsum = gamma * dot(n, f3(p) - prev);
        gamma = gamma + 1.f;
    }
    const float dL = (-C - dsum) / (gamma * im + alpha);
    const float3 dp = (-dL) * n;
    out = (-im) * dp;
    return true;
}

}  // namespace xpbd
