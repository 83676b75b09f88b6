/*
 * Bone-surface binding of muscle vertices (the reference's target_mode="mesh"
 * driver, mg/kernel.py:267-347 bone_bind_kernel / bone_slide_target_kernel,
 * driven from mg/mg.py:1117-1174).  TEST INFRASTRUCTURE ONLY: the checker of
 * csrc/xpbd_bone.cu.  FP32, brute force over all faces.
 *
 * Barycentric convention of Warp's mesh_eval_position: face f = (A, B, C),
 * position(u, v) = u A + v B + (1 - u - v) C.  The face frame follows
 * mg/kernel.py:_face_basis: p0 = position(0,0) = C, p1 = position(1,0) = A,
 * p2 = position(0,1) = B; n = normalize((p1-p0) x (p2-p0)), t1 = normalize(p1-p0),
 * t2 = n x t1, R = [t1 t2 n] (columns).
 * Closest point: the Voronoi-region walk of Ericson, Real-Time Collision
 * Detection (2005), sec. 5.1.5, restated; ties between faces keep the lowest
 * face index.
 */
#ifndef XPBD_ORACLE_BONE_H
#define XPBD_ORACLE_BONE_H

static float ob_dot(const float* a, const float* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* squared distance from p to triangle (a, b, c); *wa, *wb weights of a, b */
static float orc_closest_tri(const float* p, const float* a, const float* b, const float* c, float* wa, float* wb) {
    float ab[3], ac[3], ap[3], bp[3], cp[3];
    for (int k = 0; k < 3; ++k) {
        ab[k] = b[k] - a[k];
        ac[k] = c[k] - a[k];
        ap[k] = p[k] - a[k];
        bp[k] = p[k] - b[k];
        cp[k] = p[k] - c[k];
    }
    float u, v; /* weights of a and b */
    const float d1 = ob_dot(ab, ap), d2 = ob_dot(ac, ap);
    const float d3 = ob_dot(ab, bp), d4 = ob_dot(ac, bp);
    const float d5 = ob_dot(ab, cp), d6 = ob_dot(ac, cp);
    const float vc = d1 * d4 - d3 * d2, vb = d5 * d2 - d1 * d6, va = d3 * d6 - d5 * d4;
    if (d1 <= 0.f && d2 <= 0.f) {
        u = 1.f; v = 0.f;
    } else if (d3 >= 0.f && d4 <= d3) {
        u = 0.f; v = 1.f;
    } else if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f) {
        const float t = d1 / (d1 - d3);
        u = 1.f - t; v = t;
    } else if (d6 >= 0.f && d5 <= d6) {
        u = 0.f; v = 0.f;
    } else if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f) {
        const float t = d2 / (d2 - d6);
        u = 1.f - t; v = 0.f;
    } else if (va <= 0.f && (d4 - d3) >= 0.f && (d5 - d6) >= 0.f) {
        const float t = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        u = 0.f; v = 1.f - t;
    } else {
        const float den = 1.f / (va + vb + vc);
        const float s = vb * den, t = vc * den; /* weights of b and c */
        u = 1.f - s - t; v = s;
    }
    const float w = 1.f - u - v;
    float d = 0.f;
    for (int k = 0; k < 3; ++k) {
        const float q = u * a[k] + v * b[k] + w * c[k];
        d += (p[k] - q) * (p[k] - q);
    }
    *wa = u;
    *wb = v;
    return d;
}

static void ob_eval(const float* bp4, const int* tris, int f, float u, float v, float* out) {
    const float* A = bp4 + 4 * tris[3 * f];
    const float* B = bp4 + 4 * tris[3 * f + 1];
    const float* C = bp4 + 4 * tris[3 * f + 2];
    const float w = 1.f - u - v;
    for (int k = 0; k < 3; ++k) out[k] = u * A[k] + v * B[k] + w * C[k];
}

static void ob_norm(float* a) {
    const float l = sqrtf(ob_dot(a, a));
    const float s = l > 0.f ? 1.f / l : 0.f;
    a[0] *= s; a[1] *= s; a[2] *= s;
}

/* R[row][col], columns t1, t2, n */
static void ob_basis(const float* bp4, const int* tris, int f, float R[3][3]) {
    float p0[3], p1[3], p2[3], e1[3], e2[3], n[3], t1[3], t2[3];
    ob_eval(bp4, tris, f, 0.f, 0.f, p0);
    ob_eval(bp4, tris, f, 1.f, 0.f, p1);
    ob_eval(bp4, tris, f, 0.f, 1.f, p2);
    for (int k = 0; k < 3; ++k) { e1[k] = p1[k] - p0[k]; e2[k] = p2[k] - p0[k]; }
    n[0] = e1[1] * e2[2] - e1[2] * e2[1];
    n[1] = e1[2] * e2[0] - e1[0] * e2[2];
    n[2] = e1[0] * e2[1] - e1[1] * e2[0];
    ob_norm(n);
    for (int k = 0; k < 3; ++k) t1[k] = e1[k];
    ob_norm(t1);
    t2[0] = n[1] * t1[2] - n[2] * t1[1];
    t2[1] = n[2] * t1[0] - n[0] * t1[2];
    t2[2] = n[0] * t1[1] - n[1] * t1[0];
    for (int k = 0; k < 3; ++k) { R[k][0] = t1[k]; R[k][1] = t2[k]; R[k][2] = n[k]; }
}

/* closest face within max_dist; returns the face or -1 */
static int ob_query(const float* p, const float* bp4, int nt, const int* tris, float max_dist, float* u, float* v) {
    int best = -1;
    float bd = max_dist * max_dist;
    for (int f = 0; f < nt; ++f) {
        float a, b;
        const float d = orc_closest_tri(p, bp4 + 4 * tris[3 * f], bp4 + 4 * tris[3 * f + 1], bp4 + 4 * tris[3 * f + 2],
                                        &a, &b);
        if (d < bd || (best < 0 && d <= bd)) {
            bd = d;
            best = f;
            *u = a;
            *v = b;
        }
    }
    return best;
}

/* bone_bind_kernel (mg/kernel.py:287-310): q4 [n][4], bone4 [nbv][4], tris
 * [nt][3]; out_face [n], out_uv [n][2], out_local [n][4] (R^T (q - cp), w 0). */
void orc_bone_bind(int n, const float* q4, const float* bone4, int nt, const int* tris, float max_dist, int* out_face,
                   float* out_uv, float* out_local) {
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < n; ++i) {
        float u = 0.f, v = 0.f;
        const int f = ob_query(q4 + 4 * i, bone4, nt, tris, max_dist, &u, &v);
        float* lo = out_local + 4 * i;
        if (f < 0) {
            out_face[i] = 0;
            out_uv[2 * i] = out_uv[2 * i + 1] = 0.f;
            lo[0] = lo[1] = lo[2] = lo[3] = 0.f;
            continue;
        }
        float cp[3], R[3][3], d[3];
        ob_eval(bone4, tris, f, u, v, cp);
        ob_basis(bone4, tris, f, R);
        for (int k = 0; k < 3; ++k) d[k] = q4[4 * i + k] - cp[k];
        for (int k = 0; k < 3; ++k) lo[k] = R[0][k] * d[0] + R[1][k] * d[1] + R[2][k] * d[2];
        lo[3] = 0.f;
        out_face[i] = f;
        out_uv[2 * i] = u;
        out_uv[2 * i + 1] = v;
    }
}

/* bone_slide_target_kernel (mg/kernel.py:313-347); bind_face/bind_uv/local
 * updated in place on an accepted slide; target4[i].xyz = cp + R local. */
void orc_bone_slide_targets(int n, const float* m4, const int* anchor_face, const float* anchor_uv, int* bind_face,
                            float* bind_uv, float* local4, float slide_range, int reproject, float max_dist,
                            const float* bone4, int nt, const int* tris, float* target4) {
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < n; ++i) {
        float ap[3];
        ob_eval(bone4, tris, anchor_face[i], anchor_uv[2 * i], anchor_uv[2 * i + 1], ap);
        if (reproject) {
            float u = 0.f, v = 0.f;
            const int f = ob_query(m4 + 4 * i, bone4, nt, tris, max_dist, &u, &v);
            if (f >= 0) {
                float cand[3], dd[3];
                ob_eval(bone4, tris, f, u, v, cand);
                for (int k = 0; k < 3; ++k) dd[k] = cand[k] - ap[k];
                if (sqrtf(ob_dot(dd, dd)) <= slide_range) {
                    float R[3][3], d[3];
                    bind_face[i] = f;
                    bind_uv[2 * i] = u;
                    bind_uv[2 * i + 1] = v;
                    ob_basis(bone4, tris, f, R);
                    for (int k = 0; k < 3; ++k) d[k] = m4[4 * i + k] - cand[k];
                    for (int k = 0; k < 3; ++k) local4[4 * i + k] = R[0][k] * d[0] + R[1][k] * d[1] + R[2][k] * d[2];
                }
            }
        }
        const int f = bind_face[i];
        float cp[3], R[3][3];
        ob_eval(bone4, tris, f, bind_uv[2 * i], bind_uv[2 * i + 1], cp);
        ob_basis(bone4, tris, f, R);
        const float* l = local4 + 4 * i;
        for (int k = 0; k < 3; ++k) target4[4 * i + k] = cp[k] + (R[k][0] * l[0] + R[k][1] * l[1] + R[k][2] * l[2]);
    }
}

/* rigid pose of bone-surface vertices: out4[j] = R_b rest4[j] + t_b with
 * transforms [nb][12] row-major 3x4 [R | t], b = vert_bone[j] */
void orc_bone_pose(int nbv, const float* rest4, const int* vert_bone, const float* tr, float* out4) {
    for (int j = 0; j < nbv; ++j) {
        const float* T = tr + 12 * vert_bone[j];
        const float* x = rest4 + 4 * j;
        for (int r = 0; r < 3; ++r)
            out4[4 * j + r] = ((T[4 * r] * x[0] + T[4 * r + 1] * x[1]) + T[4 * r + 2] * x[2]) + T[4 * r + 3];
        out4[4 * j + 3] = 0.f;
    }
}

/* solve_m2m_glue_kernel (mg/kernel.py:350-394), pairs in index order, each
 * seeing the corrections of the pairs before it; pos4.w = inverse mass. */
void orc_m2m_glue(int n, const int* pa, const int* pb, const float* restlen, const float* compliance, float* pos4,
                  float dt, float omega) {
    for (int c = 0; c < n; ++c) {
        float* xa = pos4 + 4 * pa[c];
        float* xb = pos4 + 4 * pb[c];
        const float d[3] = {xa[0] - xb[0], xa[1] - xb[1], xa[2] - xb[2]};
        const float len = sqrtf(ob_dot(d, d));
        if (len < 1.0e-9f) continue;
        const float dir[3] = {d[0] / len, d[1] / len, d[2] / len};
        const float C = len - restlen[c];
        const float wa = xa[3], wb = xb[3];
        const float at = compliance[c] / (dt * dt);
        const float den = (wa + wb) + at;
        if (den < 1.0e-12f) continue;
        const float f = omega * (-C / den);
        for (int k = 0; k < 3; ++k) {
            xa[k] += (f * wa) * dir[k];
            xb[k] += (-f * wb) * dir[k];
        }
    }
}

/* fascia_bind_kernel (fascia/fascia.py:130-157): face, uv, signed normal gap
 * (q - cp) . n of the closest surface face within max_dist; ok 0 when none. */
void orc_surface_bind(int n, const float* q4, const float* surf4, int nt, const int* tris, float max_dist, int* out_face,
                      float* out_uv, float* out_gap, int* out_ok) {
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < n; ++i) {
        float u = 0.f, v = 0.f;
        const int f = ob_query(q4 + 4 * i, surf4, nt, tris, max_dist, &u, &v);
        if (f < 0) {
            out_face[i] = 0;
            out_uv[2 * i] = out_uv[2 * i + 1] = 0.f;
            out_gap[i] = 0.f;
            out_ok[i] = 0;
            continue;
        }
        float cp[3], R[3][3], d[3];
        ob_eval(surf4, tris, f, u, v, cp);
        ob_basis(surf4, tris, f, R);
        for (int k = 0; k < 3; ++k) d[k] = q4[4 * i + k] - cp[k];
        out_face[i] = f;
        out_uv[2 * i] = u;
        out_uv[2 * i + 1] = v;
        out_gap[i] = R[0][2] * d[0] + R[1][2] * d[1] + R[2][2] * d[2];
        out_ok[i] = 1;
    }
}

/* fascia_ride_kernel (fascia/fascia.py:160-176) */
void orc_surface_ride(int n, const int* bound, const int* face, const float* uv, const float* gap, const float* surf4,
                      const int* tris, float* fascia4) {
    for (int i = 0; i < n; ++i) {
        float cp[3], R[3][3];
        ob_eval(surf4, tris, face[i], uv[2 * i], uv[2 * i + 1], cp);
        ob_basis(surf4, tris, face[i], R);
        for (int k = 0; k < 3; ++k) fascia4[4 * bound[i] + k] = cp[k] + R[k][2] * gap[i];
    }
}

/* fascia_advect_bone_kernel (fascia/fascia.py:45-62) */
void orc_fascia_advect(int n, const int* follow, const float* target4, float* prev4, float* fascia4) {
    for (int i = 0; i < n; ++i) {
        const float* cur = target4 + 4 * follow[i];
        for (int k = 0; k < 3; ++k) {
            fascia4[4 * i + k] = fascia4[4 * i + k] + (cur[k] - prev4[4 * i + k]);
            prev4[4 * i + k] = cur[k];
        }
    }
}

/* fascia_anchor_bone_kernel (fascia/fascia.py:65-80) */
void orc_fascia_anchor(int n, const int* local, const int* cons, const float* offset4, const float* target4,
                       float* fascia4) {
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) fascia4[4 * local[i] + k] = target4[4 * cons[i] + k] + offset4[4 * i + k];
}

/* solve_glue_kernel (fascia/fascia.py:83-125), pairs in index order */
void orc_fascia_glue(int n, const int* pf, const int* pm, const float* restlen, const float* compliance,
                     const float* fascia4, float* muscle4, float dt, float omega) {
    for (int c = 0; c < n; ++c) {
        const float* xf = fascia4 + 4 * pf[c];
        float* xm = muscle4 + 4 * pm[c];
        const float d[3] = {xf[0] - xm[0], xf[1] - xm[1], xf[2] - xm[2]};
        const float len = sqrtf(ob_dot(d, d));
        if (len < 1.0e-9f) continue;
        const float dir[3] = {d[0] / len, d[1] / len, d[2] / len};
        const float C = len - restlen[c];
        const float wj = xm[3];
        const float at = compliance[c] / (dt * dt);
        const float den = wj + at;
        if (den < 1.0e-12f) continue;
        const float f = omega * (-C / den);
        for (int k = 0; k < 3; ++k) xm[k] += (-f * wj) * dir[k];
    }
}

#endif
