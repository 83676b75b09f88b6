/*
 * DCD part of the oracle (FP32 only, the reference's precision) -- TEST
 * INFRASTRUCTURE ONLY.  Restates collision/udcf/kernel.py of the reference:
 * tri_aabb_kernel (:917-934), the pair rules of broadphase_find_pairs_bvh_kernel
 * (:937-981) evaluated exhaustively (sweep and prune on x, so the pair SET is
 * independent of any tree), narrow_kernel (:316-474) per pair in pair order,
 * respond_kernel (:713-806) accumulated serially in contact order, and
 * apply_kernel (:809-822).
 */
#define DTHRESH 1.0e-5f

typedef struct { float x, y, z; } d3;
static inline d3 dmk(float x, float y, float z) { d3 r = {x, y, z}; return r; }
static inline d3 dld(const float* p, int i) { return dmk(p[4 * i], p[4 * i + 1], p[4 * i + 2]); }
static inline d3 dadd(d3 a, d3 b) { return dmk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline d3 dsub(d3 a, d3 b) { return dmk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline d3 dscl(float s, d3 a) { return dmk(s * a.x, s * a.y, s * a.z); }
static inline float ddot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline d3 dcross(d3 a, d3 b) { return dmk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static inline float dlen(d3 a) { return sqrtf(ddot(a, a)); }
static inline d3 dpick(d3 a, d3 b, d3 c, int i) { return i == 0 ? a : (i == 1 ? b : c); }

/* pos4: [n][4] (x, y, z, inverse mass).  boxes out: [ntri][6]. */
void orc_dcd_aabb(int ntri, const int* tris, const float* pos4, float thickness, float* boxes) {
    for (int i = 0; i < ntri; ++i) {
        d3 a = dld(pos4, tris[3 * i]), b = dld(pos4, tris[3 * i + 1]), c = dld(pos4, tris[3 * i + 2]);
        float* o = boxes + 6 * i;
        o[0] = fminf(fminf(a.x, b.x), c.x) - thickness; o[1] = fminf(fminf(a.y, b.y), c.y) - thickness;
        o[2] = fminf(fminf(a.z, b.z), c.z) - thickness; o[3] = fmaxf(fmaxf(a.x, b.x), c.x) + thickness;
        o[4] = fmaxf(fmaxf(a.y, b.y), c.y) + thickness; o[5] = fmaxf(fmaxf(a.z, b.z), c.z) + thickness;
    }
}

static int cmpll(const void* x, const void* y) {
    long long a = *(const long long*)x, b = *(const long long*)y;
    return a < b ? -1 : (a > b ? 1 : 0);
}

static const float* g_boxes;
static int cmp_lox(const void* a, const void* b) {
    float fa = g_boxes[6 * *(const int*)a], fb = g_boxes[6 * *(const int*)b];
    return fa < fb ? -1 : (fa > fb ? 1 : (*(const int*)a - *(const int*)b));
}

/* All pairs (i, j > i) with overlapping boxes that pass the group rules,
 * written sorted by (i, j).  Returns the pair count (writes at most cap). */
long orc_dcd_pairs(int ntri, const int* tris, const int* group, int allow_self, const float* boxes, int* pairs,
                   long cap) {
    int* ord = (int*)malloc(sizeof(int) * (size_t)ntri);
    for (int i = 0; i < ntri; ++i) ord[i] = i;
    g_boxes = boxes;
    qsort(ord, (size_t)ntri, sizeof(int), cmp_lox);
    long n = 0;
    /* collect candidate pairs, then sort by (i, j) */
    long pcap = 1 << 20, pn = 0;
    long long* keys = (long long*)malloc(sizeof(long long) * (size_t)pcap);
    for (int a = 0; a < ntri; ++a) {
        int i = ord[a];
        const float* A = boxes + 6 * i;
        for (int b = a + 1; b < ntri; ++b) {
            int j = ord[b];
            const float* Bx = boxes + 6 * j;
            if (Bx[0] > A[3]) break;
            if (A[1] > Bx[4] || Bx[1] > A[4] || A[2] > Bx[5] || Bx[2] > A[5]) continue;
            int lo = i < j ? i : j, hi = i < j ? j : i;
            int gi = group ? group[lo] : 0, gj = group ? group[hi] : 0;
            if (gi == 1 && gj == 1) continue;
            if (gi == 0 && gj == 0) {
                if (!allow_self) continue;
                int share = 0;
                for (int u = 0; u < 3; ++u)
                    for (int v = 0; v < 3; ++v) share |= tris[3 * lo + u] == tris[3 * hi + v];
                if (share) continue;
            }
            if (pn == pcap) { pcap *= 2; keys = (long long*)realloc(keys, sizeof(long long) * (size_t)pcap); }
            keys[pn++] = (long long)lo * ntri + hi;
        }
    }
    qsort(keys, (size_t)pn, sizeof(long long), cmpll);
    for (long k = 0; k < pn; ++k) {
        if (n < cap) { pairs[2 * n] = (int)(keys[k] / ntri); pairs[2 * n + 1] = (int)(keys[k] % ntri); }
        ++n;
    }
    free(keys);
    free(ord);
    return n;
}
static int d_inside(d3 p1, d3 p2, d3 p3, d3 p) {
    d3 c1 = dcross(dsub(p2, p1), dsub(p, p2)), c2 = dcross(dsub(p3, p2), dsub(p, p3)), c3 = dcross(dsub(p1, p3), dsub(p, p1));
    return ddot(c1, c2) > 0.f && ddot(c1, c3) > 0.f;
}
static d3 d_bary(d3 A, d3 B, d3 C, d3 P) {
    d3 v0 = dsub(B, A), v1 = dsub(C, A), v2 = dsub(P, A);
    float d00 = ddot(v0, v0), d01 = ddot(v0, v1), d11 = ddot(v1, v1), d20 = ddot(v2, v0), d21 = ddot(v2, v1);
    float den = d00 * d11 - d01 * d01;
    if (den == 0.f) return dmk(1.f / 3.f, 1.f / 3.f, 1.f / 3.f);
    float v = (d11 * d20 - d01 * d21) / den, w = (d00 * d21 - d01 * d20) / den;
    return dmk(1.f - v - w, v, w);
}
static int d_line(d3 p1, d3 p2, d3 p3, d3 p4, d3 v1, d3 v2, d3* out) {
    d3 d1 = dsub(p2, p1), d2 = dsub(p4, p3), nrm = dcross(d1, d2);
    if (dlen(nrm) < 1.0e-6f) return 0;
    float den = ddot(nrm, nrm);
    if (den < 1.0e-6f) return 0;
    d3 v = dsub(p3, p1);
    float t1 = ddot(dcross(v, d2), nrm) / den, t2 = ddot(dcross(v, d1), nrm) / den;
    if (!(t2 >= 0.f && t2 <= 1.f && t1 >= 0.f && t1 <= 1.f)) return 0;
    *out = dadd(v1, dscl(t1, dsub(v2, v1)));
    return 1;
}
static int d_gen_t(d3 N, d3 v0, d3 v1, d3 v2, float d, d3 D, float* lo, float* hi) {
    float d0 = ddot(N, v0) + d, e1 = ddot(N, v1) + d, e2 = ddot(N, v2) + d;
    if (d0 <= DTHRESH && e1 <= DTHRESH && e2 <= DTHRESH) return 0;
    if (d0 >= -DTHRESH && e1 >= -DTHRESH && e2 >= -DTHRESH) return 0;
    d3 s0 = v0, s1 = v1, s2 = v2;
    float f0 = d0, f1 = e1, f2 = e2;
    if ((d0 <= 0.f && e1 >= 0.f && e2 >= 0.f) || (d0 >= 0.f && e1 <= 0.f && e2 <= 0.f)) {
        s0 = v1; s1 = v0; f0 = e1; f1 = d0;
    } else if ((d0 >= 0.f && e1 >= 0.f && e2 <= 0.f) || (d0 <= 0.f && e1 <= 0.f && e2 >= 0.f)) {
        s1 = v2; s2 = v1; f1 = e2; f2 = e1;
    }
    float p0 = ddot(D, s0), p1 = ddot(D, s1), p2 = ddot(D, s2);
    float tA = p0 + (p1 - p0) * fabsf(f0 / (f0 - f1)), tB = p2 + (p1 - p2) * fabsf(f2 / (f2 - f1));
    *lo = tA > tB ? tB : tA;
    *hi = tA > tB ? tA : tB;
    return 1;
}

/* narrow_kernel per pair in pair order; contacts appended in that order.
 * c_ids [cap][8] (cur verts, pair, closest verts, 0), c_data [cap][12]. */
long orc_dcd_narrow(long npairs, const int* pairs, const int* tris, const float* pos4, float offset_eps, int* c_ids,
                    float* c_data, long cap) {
    long nc = 0;
    for (long k = 0; k < npairs; ++k) {
        int ta = pairs[2 * k], tb = pairs[2 * k + 1];
        d3 q00 = dld(pos4, tris[3 * ta]), q01 = dld(pos4, tris[3 * ta + 1]), q02 = dld(pos4, tris[3 * ta + 2]);
        d3 q10 = dld(pos4, tris[3 * tb]), q11 = dld(pos4, tris[3 * tb + 1]), q12 = dld(pos4, tris[3 * tb + 2]);
        d3 n1f = dcross(dsub(q01, q00), dsub(q02, q00)), n2f = dcross(dsub(q11, q10), dsub(q12, q10));
        float l1 = dlen(n1f), l2 = dlen(n2f);
        if (l1 == 0.f || l2 == 0.f) continue;
        d3 N1 = dmk(n1f.x / l1, n1f.y / l1, n1f.z / l1), N2 = dmk(n2f.x / l2, n2f.y / l2, n2f.z / l2);
        float d1 = -ddot(N1, q00), d2 = -ddot(N2, q10);
        d3 cp = dcross(N1, N2);
        float lcp = dlen(cp);
        if (lcp < 1.0e-8f) continue;
        d3 D = dmk(cp.x / lcp, cp.y / lcp, cp.z / lcp);
        float t1, t2, t3, t4;
        if (!d_gen_t(N2, q00, q01, q02, d2, D, &t1, &t2)) continue;
        if (!d_gen_t(N1, q10, q11, q12, d1, D, &t3, &t4)) continue;
        if (!(t2 >= t3 && t4 >= t1)) continue;
        float C1 = 0.f, C2 = 0.f;
        d3 b1 = dmk(0, 0, 0), b2 = b1, b3 = b1, b4 = b1;
        for (int j = 0; j < 3; ++j) {
            d3 q0j = dpick(q00, q01, q02, j), q1j = dpick(q10, q11, q12, j);
            d3 P0j = dsub(q0j, dscl(ddot(N2, dsub(q0j, q10)), N2));
            if (d_inside(q10, q11, q12, P0j)) {
                float cand = ddot(N2, q0j) + d2;
                if (C1 < -cand) { C1 = -cand; b1 = d_bary(q00, q01, q02, q0j); b2 = d_bary(q10, q11, q12, dsub(q0j, dscl(cand, N2))); }
            }
            float den = ddot(N1, N2);
            if (den != 0.f) {
                float t = ddot(N1, dsub(q00, q1j)) / den;
                d3 Q0j = dadd(q1j, dscl(t, N2));
                if (d_inside(q00, q01, q02, Q0j)) {
                    float cand = ddot(N2, Q0j) + d2;
                    if (C1 < -cand) { C1 = -cand; b1 = d_bary(q00, q01, q02, Q0j); b2 = d_bary(q10, q11, q12, dsub(Q0j, dscl(cand, N2))); }
                }
            }
            d3 P1j = dsub(q1j, dscl(ddot(N1, dsub(q1j, q00)), N1));
            if (d_inside(q00, q01, q02, P1j)) {
                float cand = ddot(N1, q1j) + d1;
                if (C2 < -cand) { C2 = -cand; b3 = d_bary(q10, q11, q12, q1j); b4 = d_bary(q00, q01, q02, dsub(q1j, dscl(cand, N1))); }
            }
            den = ddot(N2, N1);
            if (den != 0.f) {
                float t = ddot(N2, dsub(q10, q0j)) / den;
                d3 Q1j = dadd(q0j, dscl(t, N1));
                if (d_inside(q10, q11, q12, Q1j)) {
                    float cand = ddot(N1, Q1j) + d1;
                    if (C2 < -cand) { C2 = -cand; b3 = d_bary(q10, q11, q12, Q1j); b4 = d_bary(q00, q01, q02, dsub(Q1j, dscl(cand, N1))); }
                }
            }
            int jn = (j + 1) % 3;
            d3 q0jn = dpick(q00, q01, q02, jn), q1jn = dpick(q10, q11, q12, jn);
            d3 P0jn = dsub(q0jn, dscl(ddot(N2, dsub(q0jn, q10)), N2));
            d3 P1jn = dsub(q1jn, dscl(ddot(N1, dsub(q1jn, q00)), N1));
            for (int kk = 0; kk < 3; ++kk) {
                int kn = (kk + 1) % 3;
                d3 o;
                if (d_line(P0j, P0jn, dpick(q10, q11, q12, kk), dpick(q10, q11, q12, kn), q0j, q0jn, &o)) {
                    float cand = ddot(N2, o) + d2;
                    if (C1 < -cand) { C1 = -cand; b1 = d_bary(q00, q01, q02, o); b2 = d_bary(q10, q11, q12, dsub(o, dscl(cand, N2))); }
                }
                if (d_line(P1j, P1jn, dpick(q00, q01, q02, kk), dpick(q00, q01, q02, kn), q1j, q1jn, &o)) {
                    float cand = ddot(N1, o) + d1;
                    if (C2 < -cand) { C2 = -cand; b3 = d_bary(q10, q11, q12, o); b4 = d_bary(q00, q01, q02, dsub(o, dscl(cand, N1))); }
                }
            }
        }
        if (C1 <= offset_eps || C2 <= offset_eps) continue;
        if (nc < cap) {
            int first = C1 < C2;
            int tc = first ? ta : tb, tl = first ? tb : ta;
            int* ci = c_ids + 8 * nc;
            ci[0] = tris[3 * tc]; ci[1] = tris[3 * tc + 1]; ci[2] = tris[3 * tc + 2]; ci[3] = (int)k;
            ci[4] = tris[3 * tl]; ci[5] = tris[3 * tl + 1]; ci[6] = tris[3 * tl + 2]; ci[7] = 0;
            d3 n = first ? N2 : N1, bb1 = first ? b1 : b3, bb2 = first ? b2 : b4;
            float* cf = c_data + 12 * nc;
            cf[0] = n.x; cf[1] = n.y; cf[2] = n.z; cf[3] = first ? C1 : C2;
            cf[4] = bb1.x; cf[5] = bb1.y; cf[6] = bb1.z; cf[7] = C1;
            cf[8] = bb2.x; cf[9] = bb2.y; cf[10] = bb2.z; cf[11] = C2;
        }
        ++nc;
    }
    return nc;
}

/* respond_kernel accumulated serially into dP4 ([n][4] dP.xyz, count), then
 * apply_kernel onto pos4 (clears dP4). */
void orc_dcd_respond_apply(long nc, const int* c_ids, const float* c_data, float* pos4, const float* xprev4, int nverts,
                           float multiplier, float mu_s, float mu_d, float max_push, int jacobi_avg, float* dP4) {
    for (long k = 0; k < nc; ++k) {
        const int* ci = c_ids + 8 * k;
        const float* cf = c_data + 12 * k;
        float pen = cf[3];
        if (max_push > 0.f && pen > max_push) pen = max_push;
        float C = pen * multiplier;
        if (C == 0.f) continue;
        d3 nrm = dmk(cf[0], cf[1], cf[2]);
        int cu[3] = {ci[0], ci[1], ci[2]}, cl[3] = {ci[4], ci[5], ci[6]};
        int solid_cur = pos4[4 * cu[0] + 3] == 0.f || pos4[4 * cu[1] + 3] == 0.f || pos4[4 * cu[2] + 3] == 0.f;
        int solid_clo = pos4[4 * cl[0] + 3] == 0.f || pos4[4 * cl[1] + 3] == 0.f || pos4[4 * cl[2] + 3] == 0.f;
        if (!solid_cur && !solid_clo) C = C * 0.5f;
        d3 push_clo = solid_clo ? dmk(0, 0, 0) : dscl(-C, nrm);
        d3 push_cur = solid_cur ? dmk(0, 0, 0) : dscl(C, nrm);
        d3 v[6];
        for (int m = 0; m < 3; ++m) {
            v[m] = dsub(dadd(dld(pos4, cl[m]), push_clo), dld(xprev4, cl[m]));
            v[3 + m] = dsub(dadd(dld(pos4, cu[m]), push_cur), dld(xprev4, cu[m]));
        }
        float ln = dlen(nrm);
        d3 g = dmk(nrm.x / ln, nrm.y / ln, nrm.z / ln);
        d3 vclo = dadd(dadd(dscl(cf[4], v[0]), dscl(cf[5], v[1])), dscl(cf[6], v[2]));
        d3 perp_clo = dsub(vclo, dscl(ddot(vclo, g), g));
        d3 vcur = dadd(dadd(dscl(cf[8], v[3]), dscl(cf[9], v[4])), dscl(cf[10], v[5]));
        d3 perp_cur = dsub(vcur, dscl(ddot(vcur, g), g));
        d3 diff = dsub(perp_cur, perp_clo);
        float dn = dlen(diff);
        if (dn > pen * mu_s && dn > 0.f) diff = dscl(pen * mu_d / dn, diff);
        d3 diffV = dscl(0.5f, diff), diffT = dsub(diff, diffV);
        d3 mu_ = dsub(push_cur, diffV), ml = dadd(push_clo, diffT);
        for (int m = 0; m < 3; ++m) {
            if (pos4[4 * cu[m] + 3] > 0.f) {
                float* a = dP4 + 4 * cu[m];
                a[0] += mu_.x; a[1] += mu_.y; a[2] += mu_.z; a[3] += 1.f;
            }
            if (pos4[4 * cl[m] + 3] > 0.f) {
                float* a = dP4 + 4 * cl[m];
                a[0] += ml.x; a[1] += ml.y; a[2] += ml.z; a[3] += 1.f;
            }
        }
    }
    for (int i = 0; i < nverts; ++i) {
        float* a = dP4 + 4 * i;
        if (a[3] > 0.f) {
            if (jacobi_avg) {
                pos4[4 * i] += a[0] / a[3]; pos4[4 * i + 1] += a[1] / a[3]; pos4[4 * i + 2] += a[2] / a[3];
            } else {
                pos4[4 * i] += a[0]; pos4[4 * i + 1] += a[1]; pos4[4 * i + 2] += a[2];
            }
            a[0] = a[1] = a[2] = a[3] = 0.f;
        }
    }
}
