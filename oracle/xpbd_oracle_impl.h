/*
 * XPBD oracle, precision-generic body.  TEST INFRASTRUCTURE ONLY.
 *
 * This file is included twice by xpbd_oracle.c, once with REAL=float (suffix
 * _f32) and once with REAL=double (suffix _f64).  It restates, kernel by
 * kernel, the arithmetic of the reference solver (chunleili/rlmuscleV2,
 * src/muscle/...) in plain C, in the reference's operation order, so that it
 * can serve as the parity checker of the CUDA path.  Nothing in the product
 * links or calls this code.
 *
 * Jacobi accumulation order: the reference scatters with float atomics, so its
 * order is not defined.  The oracle fixes one: every vertex sums the
 * corrections of its incident constraints in constraint-table order (the
 * table is sorted by ConstraintType tag, as in engine.py:1179 /
 * musclesim.py:370).  Phase A computes all corrections in parallel, phase B
 * sums them per vertex through a CSR adjacency; the result is bitwise equal to
 * a serial scatter in table order, independent of the thread count.
 */

#define CAT2(a, b) a##_##b
#define CAT(a, b) CAT2(a, b)
#define FN(name) CAT(name, SFX)
#define VEC FN(vec)
#define MAT FN(mat)

typedef struct { REAL x, y, z; } VEC;
typedef struct { REAL m[3][3]; } MAT;

static inline VEC FN(mk)(REAL x, REAL y, REAL z) { VEC r; r.x = x; r.y = y; r.z = z; return r; }
static inline VEC FN(ld)(const REAL* p, long i) { return FN(mk)(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }
static inline void FN(st)(REAL* p, long i, VEC v) { p[3 * i] = v.x; p[3 * i + 1] = v.y; p[3 * i + 2] = v.z; }
static inline VEC FN(add)(VEC a, VEC b) { return FN(mk)(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline VEC FN(sub)(VEC a, VEC b) { return FN(mk)(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline VEC FN(neg)(VEC a) { return FN(mk)(-a.x, -a.y, -a.z); }
static inline VEC FN(scl)(REAL s, VEC a) { return FN(mk)(s * a.x, s * a.y, s * a.z); }
static inline VEC FN(dvs)(VEC a, REAL s) { return FN(mk)(a.x / s, a.y / s, a.z / s); }
static inline REAL FN(dot)(VEC a, VEC b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline VEC FN(cross)(VEC a, VEC b) {
    return FN(mk)(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline REAL FN(len)(VEC a) { return (REAL)sqrt((double)FN(dot)(a, a)); }
#define SQRT(v) ((REAL)sqrt((double)(v)))

/* Ds with columns c0,c1,c2 (engine.py:209-213 layout). */
static inline MAT FN(cols)(VEC c0, VEC c1, VEC c2) {
    MAT M;
    M.m[0][0] = c0.x; M.m[0][1] = c1.x; M.m[0][2] = c2.x;
    M.m[1][0] = c0.y; M.m[1][1] = c1.y; M.m[1][2] = c2.y;
    M.m[2][0] = c0.z; M.m[2][1] = c1.z; M.m[2][2] = c2.z;
    return M;
}
static inline MAT FN(mul)(MAT A, MAT B) {
    MAT C;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            C.m[i][j] = A.m[i][0] * B.m[0][j] + A.m[i][1] * B.m[1][j] + A.m[i][2] * B.m[2][j];
    return C;
}
static inline REAL FN(det)(MAT M) {
    return M.m[0][0] * (M.m[1][1] * M.m[2][2] - M.m[1][2] * M.m[2][1])
         - M.m[0][1] * (M.m[1][0] * M.m[2][2] - M.m[1][2] * M.m[2][0])
         + M.m[0][2] * (M.m[1][0] * M.m[2][1] - M.m[1][1] * M.m[2][0]);
}
static inline MAT FN(ldB)(const REAL* B, long t) {
    MAT M;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) M.m[i][j] = B[9 * t + 3 * i + j];
    return M;
}
/* grad_k[a] = sum_j dCdF[a][j] * B[k][j]  (solve_kernels.py:1276-1288). */
static inline VEC FN(gradrow)(MAT G, MAT B, int k) {
    return FN(mk)(G.m[0][0] * B.m[k][0] + G.m[0][1] * B.m[k][1] + G.m[0][2] * B.m[k][2],
                  G.m[1][0] * B.m[k][0] + G.m[1][1] * B.m[k][1] + G.m[1][2] * B.m[k][2],
                  G.m[2][0] * B.m[k][0] + G.m[2][1] * B.m[k][1] + G.m[2][2] * B.m[k][2]);
}

/* get_inv_mass_fn, solve_kernels.py:71-80. */
static inline REAL FN(invm)(const REAL* mass, const int* stopped, int i) {
    if (stopped[i] != 0) return (REAL)0;
    REAL m = mass[i];
    return m > (REAL)0 ? (REAL)1 / m : (REAL)0;
}

/* ------------------------------------------------------------------------ */
/* Sign-fixed SVD (ssvd_fn, solve_kernels.py:85-112).  The reference calls
 * Warp's svd3 and then forces det(U)=det(V)=+1 by negating the last column
 * and the last singular value.  The resulting factorisation is: U, V
 * rotations, |s0|>=|s1|>=|s2|, s0,s1>=0, sign(s2)=sign(det F).  The oracle
 * computes that factorisation to double precision: cyclic Jacobi on F^T F
 * (Golub & Van Loan, sec. 8.5) run to convergence, eigenvalues sorted
 * descending, then u0=F v0/|F v0|, u1 by Gram-Schmidt, u2=u0 x u1 and
 * s2=u2.(F v2). */
void FN(orc_svd3)(const REAL* Fin, REAL* Uout, REAL* sout, REAL* Vout) {
    double F[3][3], S[3][3], V[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) F[i][j] = (double)Fin[3 * i + j];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            S[i][j] = F[0][i] * F[0][j] + F[1][i] * F[1][j] + F[2][i] * F[2][j];
            V[i][j] = (i == j) ? 1.0 : 0.0;
        }
    for (int sweep = 0; sweep < 64; ++sweep) {
        double off = S[0][1] * S[0][1] + S[0][2] * S[0][2] + S[1][2] * S[1][2];
        double dia = S[0][0] * S[0][0] + S[1][1] * S[1][1] + S[2][2] * S[2][2];
        if (off <= 1e-36 * dia || off == 0.0) break;
        for (int pq = 0; pq < 3; ++pq) {
            int p = (pq == 2) ? 1 : 0, q = (pq == 0) ? 1 : 2;
            double apq = S[p][q];
            if (apq == 0.0) continue;
            double theta = (S[q][q] - S[p][p]) / (2.0 * apq);
            double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
            double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
            for (int k = 0; k < 3; ++k) { /* S <- S J */
                double skp = S[k][p], skq = S[k][q];
                S[k][p] = c * skp - s * skq;
                S[k][q] = s * skp + c * skq;
            }
            for (int k = 0; k < 3; ++k) { /* S <- J^T S */
                double spk = S[p][k], sqk = S[q][k];
                S[p][k] = c * spk - s * sqk;
                S[q][k] = s * spk + c * sqk;
            }
            for (int k = 0; k < 3; ++k) {
                double vkp = V[k][p], vkq = V[k][q];
                V[k][p] = c * vkp - s * vkq;
                V[k][q] = s * vkp + c * vkq;
            }
        }
    }
    double lam[3] = {S[0][0], S[1][1], S[2][2]};
    int ord[3] = {0, 1, 2};
    for (int a = 0; a < 3; ++a)
        for (int b = a + 1; b < 3; ++b)
            if (lam[ord[b]] > lam[ord[a]]) { int tmp = ord[a]; ord[a] = ord[b]; ord[b] = tmp; }
    double v[3][3]; /* v[k] = k-th column */
    for (int k = 0; k < 3; ++k)
        for (int i = 0; i < 3; ++i) v[k][i] = V[i][ord[k]];
    double dv = v[0][0] * (v[1][1] * v[2][2] - v[1][2] * v[2][1]) - v[1][0] * (v[0][1] * v[2][2] - v[0][2] * v[2][1])
              + v[2][0] * (v[0][1] * v[1][2] - v[0][2] * v[1][1]);
    if (dv < 0) for (int i = 0; i < 3; ++i) v[2][i] = -v[2][i];
    double b[3][3];
    for (int k = 0; k < 3; ++k)
        for (int i = 0; i < 3; ++i) b[k][i] = F[i][0] * v[k][0] + F[i][1] * v[k][1] + F[i][2] * v[k][2];
    double u[3][3], sg[3];
    double n0 = sqrt(b[0][0] * b[0][0] + b[0][1] * b[0][1] + b[0][2] * b[0][2]);
    if (n0 > 1e-300) { for (int i = 0; i < 3; ++i) u[0][i] = b[0][i] / n0; }
    else { u[0][0] = 1; u[0][1] = 0; u[0][2] = 0; }
    sg[0] = n0;
    double pr = u[0][0] * b[1][0] + u[0][1] * b[1][1] + u[0][2] * b[1][2];
    double w[3] = {b[1][0] - pr * u[0][0], b[1][1] - pr * u[0][1], b[1][2] - pr * u[0][2]};
    double n1 = sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
    if (n1 > 1e-300 * (n0 > 1 ? n0 : 1)) { for (int i = 0; i < 3; ++i) u[1][i] = w[i] / n1; }
    else { /* any unit vector orthogonal to u0 */
        double a0 = fabs(u[0][0]), a1 = fabs(u[0][1]), a2 = fabs(u[0][2]);
        double e[3] = {0, 0, 0};
        if (a0 <= a1 && a0 <= a2) e[0] = 1; else if (a1 <= a2) e[1] = 1; else e[2] = 1;
        double c[3] = {u[0][1] * e[2] - u[0][2] * e[1], u[0][2] * e[0] - u[0][0] * e[2], u[0][0] * e[1] - u[0][1] * e[0]};
        double cn = sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
        for (int i = 0; i < 3; ++i) u[1][i] = c[i] / cn;
    }
    sg[1] = u[1][0] * b[1][0] + u[1][1] * b[1][1] + u[1][2] * b[1][2];
    u[2][0] = u[0][1] * u[1][2] - u[0][2] * u[1][1];
    u[2][1] = u[0][2] * u[1][0] - u[0][0] * u[1][2];
    u[2][2] = u[0][0] * u[1][1] - u[0][1] * u[1][0];
    sg[2] = u[2][0] * b[2][0] + u[2][1] * b[2][1] + u[2][2] * b[2][2];
    for (int i = 0; i < 3; ++i)
        for (int k = 0; k < 3; ++k) {
            Uout[3 * i + k] = (REAL)u[k][i];
            Vout[3 * i + k] = (REAL)v[k][i];
        }
    for (int k = 0; k < 3; ++k) sout[k] = (REAL)sg[k];
}

static inline void FN(svdm)(MAT F, MAT* U, VEC* s, MAT* V) {
    REAL f[9], u[9], sv[3], vv[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) f[3 * i + j] = F.m[i][j];
    FN(orc_svd3)(f, u, sv, vv);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) { U->m[i][j] = u[3 * i + j]; V->m[i][j] = vv[3 * i + j]; }
    *s = FN(mk)(sv[0], sv[1], sv[2]);
}

/* ------------------------------------------------------------------------ */
/* precompute_rest_kernel, engine.py:199-224 (serial, tet order). */
void FN(orc_precompute_rest)(int nt, const REAL* pos0, const int* tets, REAL density,
                             REAL* rest_volume, REAL* rest_matrix, REAL* mass, REAL* total_rest_volume) {
    for (int c = 0; c < nt; ++c) {
        const int* p = tets + 4 * c;
        VEC c0 = FN(sub)(FN(ld)(pos0, p[0]), FN(ld)(pos0, p[3]));
        VEC c1 = FN(sub)(FN(ld)(pos0, p[1]), FN(ld)(pos0, p[3]));
        VEC c2 = FN(sub)(FN(ld)(pos0, p[2]), FN(ld)(pos0, p[3]));
        MAT Dm = FN(cols)(c0, c1, c2);
        REAL d = FN(det)(Dm);
        REAL vol = (d < 0 ? -d : d) / (REAL)6;
        rest_volume[c] = vol;
        total_rest_volume[0] += vol;
        REAL mc = vol * density / (REAL)4;
        for (int i = 0; i < 4; ++i) mass[p[i]] += mc;
        /* inverse(Dm) = adjugate * (1/det) */
        REAL* B = rest_matrix + 9 * c;
        if (d != (REAL)0) {
            REAL inv = (REAL)1 / d;
            const REAL(*m)[3] = Dm.m;
            B[0] = (m[1][1] * m[2][2] - m[1][2] * m[2][1]) * inv;
            B[1] = (m[0][2] * m[2][1] - m[0][1] * m[2][2]) * inv;
            B[2] = (m[0][1] * m[1][2] - m[0][2] * m[1][1]) * inv;
            B[3] = (m[1][2] * m[2][0] - m[1][0] * m[2][2]) * inv;
            B[4] = (m[0][0] * m[2][2] - m[0][2] * m[2][0]) * inv;
            B[5] = (m[0][2] * m[1][0] - m[0][0] * m[1][2]) * inv;
            B[6] = (m[1][0] * m[2][1] - m[1][1] * m[2][0]) * inv;
            B[7] = (m[0][1] * m[2][0] - m[0][0] * m[2][1]) * inv;
            B[8] = (m[0][0] * m[1][1] - m[0][1] * m[1][0]) * inv;
        } else {
            for (int k = 0; k < 9; ++k) B[k] = 0;
        }
    }
}

/* integrate_kernel, engine.py:431-464. force may be NULL (all zero). */
void FN(orc_integrate)(int nv, REAL* pos, REAL* pprev, REAL* vel, const REAL* force, const REAL* mass,
                       const int* stopped, const REAL* g, REAL veldamping, REAL dt, int quasi_static) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nv; ++i) {
        if (stopped[i] != 0) {
            FN(st)(pprev, i, FN(ld)(pos, i));
            FN(st)(vel, i, FN(mk)(0, 0, 0));
            continue;
        }
        VEC ext = FN(mk)(g[0], g[1], g[2]);
        REAL m = mass[i];
        if (m > (REAL)1.0e-12 && force) ext = FN(add)(ext, FN(dvs)(FN(ld)(force, i), m));
        VEC p = FN(ld)(pos, i);
        FN(st)(pprev, i, p);
        if (quasi_static) {
            FN(st)(pos, i, FN(add)(p, FN(scl)(dt * dt, ext)));
            FN(st)(vel, i, FN(mk)(0, 0, 0));
        } else {
            VEC v = FN(scl)((REAL)1 - veldamping, FN(ld)(vel, i));
            v = FN(add)(v, FN(scl)(dt, ext));
            FN(st)(vel, i, v);
            FN(st)(pos, i, FN(add)(p, FN(scl)(dt, v)));
        }
    }
}

/* update_velocities_kernel (exp_damp=1, const_damp=0), engine.py:582-605. */
void FN(orc_update_velocities)(int nv, const REAL* pos, const REAL* pprev, REAL* vel, REAL dt) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nv; ++i) FN(st)(vel, i, FN(dvs)(FN(sub)(FN(ld)(pos, i), FN(ld)(pprev, i)), dt));
}

/* apply_dP_kernel, engine.py:689-698.  omega scales the averaged correction
 * (omega=1 is the reference; the reference has no relaxation factor here). */
void FN(orc_apply_dP)(int nv, REAL* pos, const REAL* dP, const REAL* dPw, REAL omega) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nv; ++i) {
        REAL w = dPw[i];
        if (w > (REAL)1e-9) {
            VEC d = FN(dvs)(FN(ld)(dP, i), w);
            if (omega != (REAL)1) d = FN(scl)(omega, d);
            FN(st)(pos, i, FN(add)(FN(ld)(pos, i), d));
        }
    }
}

/* pintotarget_overwrite_masked_kernel, mg/kernel.py:211-225. */
void FN(orc_pin_overwrite_masked)(int n, const int* pts, const REAL* target, const REAL* rest_offset,
                                  const int* active, REAL* pos) {
    for (int i = 0; i < n; ++i) {
        if (active && active[i] == 0) continue;
        FN(st)(pos, pts[i], FN(add)(FN(ld)(target, i), FN(ld)(rest_offset, i)));
    }
}

/* ------------------------------------------------------------------------ */
/* Per-constraint Jacobi corrections.  Writes up to 4 (vertex, delta) terms
 * into out (4 x 3 REAL) and a bit mask of which slots called update_dP.
 * Constraint types are the ConstraintType tags of defs.py:20-36. */
#define T_ATTACH 1650556
#define T_TETVOLUME (-215389979)
#define T_TETARAPSVD (-92199132)
#define T_TETARAPANISO (-92199133)
#define T_TETSNH (-503462311)

typedef struct {
    int nv;
    const REAL* pos; const REAL* pprev; const REAL* mass; const int* stopped;
    const REAL* rest_matrix; const REAL* v_fiber; const REAL* activation; const REAL* tendonmask;
    const int* c_type; const int* c_pts; const REAL* c_stiffness; const REAL* c_damp; const int* c_tetid;
    const REAL* c_restlength; const REAL* c_restvector; const REAL* c_restdir;
    REAL dt, contraction_ratio, fiber_stiffness_scale;
} FN(ctx);

/* ARAP-SVD skip threshold on sum((sigma-1)^2): the reference's 1e-12 unless a
 * parity test disables it (orc_set_arap_skip; the CUDA path's
 * XpbdParams.arap_skip_ssq < 0) to compare both sides without the FP32
 * rounding decision it makes on near-rest tets. */
static REAL FN(arap_skip) = (REAL)1.0e-12;
void FN(orc_set_arap_skip)(double v) { FN(arap_skip) = v == 0.0 ? (REAL)1.0e-12 : (v < 0.0 ? (REAL)1.0e-38 : (REAL)v); }

static int FN(con_arapsvd)(const FN(ctx) * X, int c, REAL out[4][3]) {
    REAL k = X->c_stiffness[c];
    if (k <= (REAL)0) return 0;
    const int* p = X->c_pts + 4 * c;
    int tid = X->c_tetid[c];
    VEC p0 = FN(ld)(X->pos, p[0]), p1 = FN(ld)(X->pos, p[1]), p2 = FN(ld)(X->pos, p[2]), p3 = FN(ld)(X->pos, p[3]);
    REAL im[4];
    for (int i = 0; i < 4; ++i) im[i] = FN(invm)(X->mass, X->stopped, p[i]);
    MAT B = FN(ldB)(X->rest_matrix, tid);
    MAT F = FN(mul)(FN(cols)(FN(sub)(p0, p3), FN(sub)(p1, p3), FN(sub)(p2, p3)), B);
    MAT U, V; VEC s;
    FN(svdm)(F, &U, &s, &V);
    VEC sm1 = FN(mk)(s.x - (REAL)1, s.y - (REAL)1, s.z - (REAL)1);
    REAL ssq = sm1.x * sm1.x + sm1.y * sm1.y + sm1.z * sm1.z;
    if (ssq < FN(arap_skip)) return 0;
    REAL C = SQRT(ssq);
    REAL invC = (REAL)1 / C;
    REAL d0 = invC * sm1.x, d1 = invC * sm1.y, d2 = invC * sm1.z;
    MAT G;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            G.m[i][j] = U.m[i][0] * V.m[j][0] * d0 + U.m[i][1] * V.m[j][1] * d1 + U.m[i][2] * V.m[j][2] * d2;
    VEC g[4];
    g[0] = FN(gradrow)(G, B, 0); g[1] = FN(gradrow)(G, B, 1); g[2] = FN(gradrow)(G, B, 2);
    g[3] = FN(sub)(FN(sub)(FN(neg)(g[0]), g[1]), g[2]);
    REAL wsum = im[0] * FN(dot)(g[0], g[0]) + im[1] * FN(dot)(g[1], g[1]) + im[2] * FN(dot)(g[2], g[2]) + im[3] * FN(dot)(g[3], g[3]);
    if (wsum == (REAL)0) return 0;
    REAL alpha = (REAL)1 / k;
    REAL at = alpha / (X->dt * X->dt);
    REAL dL = -(C + at * (REAL)0) / (wsum + at);
    for (int i = 0; i < 4; ++i) {
        VEC d = FN(scl)(dL * im[i], g[i]);
        out[i][0] = d.x; out[i][1] = d.y; out[i][2] = d.z;
    }
    return 0xF;
}

static int FN(con_volume)(const FN(ctx) * X, int c, REAL out[4][3]) {
    REAL k = X->c_stiffness[c];
    if (k <= (REAL)0) return 0;
    const int* p = X->c_pts + 4 * c;
    REAL im[4];
    for (int i = 0; i < 4; ++i) im[i] = FN(invm)(X->mass, X->stopped, p[i]);
    VEC p0 = FN(ld)(X->pos, p[0]), p1 = FN(ld)(X->pos, p[1]), p2 = FN(ld)(X->pos, p[2]), p3 = FN(ld)(X->pos, p[3]);
    VEC d0 = FN(sub)(p0, p3), d1 = FN(sub)(p1, p3), d2 = FN(sub)(p2, p3);
    VEC g[4];
    g[0] = FN(dvs)(FN(cross)(d1, d2), (REAL)6);
    g[1] = FN(dvs)(FN(cross)(d2, d0), (REAL)6);
    g[2] = FN(dvs)(FN(cross)(d0, d1), (REAL)6);
    g[3] = FN(neg)(FN(add)(FN(add)(g[0], g[1]), g[2]));
    REAL ws = im[0] * FN(dot)(g[0], g[0]) + im[1] * FN(dot)(g[1], g[1]) + im[2] * FN(dot)(g[2], g[2]) + im[3] * FN(dot)(g[3], g[3]);
    if (!(ws > (REAL)1e-9)) return 0;
    REAL volume = FN(dot)(FN(cross)(d0, d1), d2) / (REAL)6;
    REAL alpha = (REAL)1 / k;
    alpha = alpha / (X->dt * X->dt);
    REAL C = volume - X->c_restlength[c];
    REAL dsum = 0, gamma = 1;
    REAL kd = X->c_damp[c];
    if (kd > (REAL)0) {
        REAL beta = k * kd * X->dt * X->dt;
        gamma = alpha * beta / X->dt;
        VEC pp[4] = {p0, p1, p2, p3};
        dsum = 0;
        for (int i = 0; i < 4; ++i) dsum += FN(dot)(g[i], FN(sub)(pp[i], FN(ld)(X->pprev, p[i])));
        dsum = dsum * gamma;
        gamma = gamma + (REAL)1;
    }
    REAL dl = (-C - alpha * (REAL)0 - dsum) / (gamma * ws + alpha);
    for (int i = 0; i < 4; ++i) {
        VEC d = FN(scl)(dl * im[i], g[i]);
        out[i][0] = d.x; out[i][1] = d.y; out[i][2] = d.z;
    }
    return 0xF;
}

static int FN(con_aniso)(const FN(ctx) * X, int c, REAL out[4][3]) {
    REAL k = X->c_stiffness[c];
    if (k <= (REAL)0) return 0;
    const int* p = X->c_pts + 4 * c;
    int tid = X->c_tetid[c];
    VEC f0 = FN(add)(FN(add)(FN(add)(FN(ld)(X->v_fiber, p[0]), FN(ld)(X->v_fiber, p[1])), FN(ld)(X->v_fiber, p[2])),
                     FN(ld)(X->v_fiber, p[3]));
    f0 = FN(dvs)(f0, (REAL)4);
    REAL fn = FN(len)(f0);
    if (fn < (REAL)1.0e-9) return 0;
    f0 = FN(dvs)(f0, fn);
    VEC p3 = FN(ld)(X->pos, p[3]);
    VEC c0 = FN(sub)(FN(ld)(X->pos, p[0]), p3), c1 = FN(sub)(FN(ld)(X->pos, p[1]), p3), c2 = FN(sub)(FN(ld)(X->pos, p[2]), p3);
    MAT B = FN(ldB)(X->rest_matrix, tid);
    MAT F = FN(mul)(FN(cols)(c0, c1, c2), B);
    VEC d = FN(mk)(F.m[0][0] * f0.x + F.m[0][1] * f0.y + F.m[0][2] * f0.z,
                   F.m[1][0] * f0.x + F.m[1][1] * f0.y + F.m[1][2] * f0.z,
                   F.m[2][0] * f0.x + F.m[2][1] * f0.y + F.m[2][2] * f0.z);
    REAL s = FN(len)(d);
    if (s < (REAL)1.0e-9) return 0;
    REAL detF = FN(det)(F);
    if (detF <= (REAL)0 || s > (REAL)1.5) return 0;
    REAL SI4 = detF < (REAL)0 ? (REAL)-1 : (REAL)1;
    REAL belly = (REAL)1 - X->tendonmask[tid];
    REAL fiberscale = (REAL)1 - belly * X->activation[tid] * X->contraction_ratio;
    REAL diff = s - SI4 * fiberscale;
    REAL C = (REAL)0.5 * diff * diff;
    REAL gs = diff / s;
    MAT G;
    REAL dd[3] = {d.x, d.y, d.z}, ff[3] = {f0.x, f0.y, f0.z};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) G.m[i][j] = gs * (dd[i] * ff[j]);
    VEC g[4];
    g[0] = FN(gradrow)(G, B, 0); g[1] = FN(gradrow)(G, B, 1); g[2] = FN(gradrow)(G, B, 2);
    g[3] = FN(sub)(FN(sub)(FN(neg)(g[0]), g[1]), g[2]);
    REAL im[4];
    for (int i = 0; i < 4; ++i) im[i] = FN(invm)(X->mass, X->stopped, p[i]);
    REAL wsum = im[0] * FN(dot)(g[0], g[0]) + im[1] * FN(dot)(g[1], g[1]) + im[2] * FN(dot)(g[2], g[2]) + im[3] * FN(dot)(g[3], g[3]);
    if (wsum < (REAL)1.0e-20) return 0;
    REAL sv = k * X->fiber_stiffness_scale;
    REAL at = ((REAL)1 / sv) / (X->dt * X->dt);
    REAL dL = -(C + at * (REAL)0) / (wsum + at);
    for (int i = 0; i < 4; ++i) {
        VEC dv = FN(scl)(dL * im[i], g[i]);
        out[i][0] = dv.x; out[i][1] = dv.y; out[i][2] = dv.z;
    }
    return 0xF;
}

static int FN(con_snh)(const FN(ctx) * X, int c, REAL out[4][3]) {
    REAL mu = X->c_stiffness[c];
    if (mu <= (REAL)0) return 0;
    const int* p = X->c_pts + 4 * c;
    int tid = X->c_tetid[c];
    REAL lam = X->c_restdir[3 * c];
    REAL restvolume = X->c_restlength[c];
    REAL kd = X->c_damp[c];
    VEC P[4];
    REAL im[4];
    for (int i = 0; i < 4; ++i) { P[i] = FN(ld)(X->pos, p[i]); im[i] = FN(invm)(X->mass, X->stopped, p[i]); }
    VEC c0 = FN(sub)(P[0], P[3]), c1 = FN(sub)(P[1], P[3]), c2 = FN(sub)(P[2], P[3]);
    MAT B = FN(ldB)(X->rest_matrix, tid);
    MAT F = FN(mul)(FN(cols)(c0, c1, c2), B);
    REAL Ic = 0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Ic += F.m[i][j] * F.m[i][j];
    REAL rs = SQRT(Ic > (REAL)1.0e-12 ? Ic : (REAL)1.0e-12);
    REAL dC = rs - (REAL)1.7320508075688772;
    if (rs < (REAL)1.0e-6) return 0;
    REAL inv_rs = (REAL)1 / rs;
    MAT Fn;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Fn.m[i][j] = F.m[i][j] * inv_rs;
    VEC dg[4], hg[4];
    for (int kk = 0; kk < 3; ++kk)
        dg[kk] = FN(mk)(B.m[kk][0] * Fn.m[0][0] + B.m[kk][1] * Fn.m[0][1] + B.m[kk][2] * Fn.m[0][2],
                        B.m[kk][0] * Fn.m[1][0] + B.m[kk][1] * Fn.m[1][1] + B.m[kk][2] * Fn.m[1][2],
                        B.m[kk][0] * Fn.m[2][0] + B.m[kk][1] * Fn.m[2][1] + B.m[kk][2] * Fn.m[2][2]);
    dg[3] = FN(sub)(FN(sub)(FN(neg)(dg[0]), dg[1]), dg[2]);
    REAL dsw = 0;
    for (int i = 0; i < 4; ++i) dsw += im[i] * FN(dot)(dg[i], dg[i]);
    if (dsw == (REAL)0) return 0;
    REAL asnh = (REAL)1 + mu / lam;
    REAL J = FN(det)(F);
    REAL hC = J - asnh;
    REAL av6 = (restvolume < 0 ? -restvolume : restvolume) * (REAL)6;
    REAL inv_detDm = (REAL)1 / (av6 > (REAL)1.0e-20 ? av6 : (REAL)1.0e-20);
    hg[0] = FN(scl)(inv_detDm, FN(cross)(c1, c2));
    hg[1] = FN(scl)(inv_detDm, FN(cross)(c2, c0));
    hg[2] = FN(scl)(inv_detDm, FN(cross)(c0, c1));
    hg[3] = FN(sub)(FN(sub)(FN(neg)(hg[0]), hg[1]), hg[2]);
    REAL hsw = 0, dh = 0;
    for (int i = 0; i < 4; ++i) hsw += im[i] * FN(dot)(hg[i], hg[i]);
    if (hsw == (REAL)0) return 0;
    for (int i = 0; i < 4; ++i) dh += im[i] * FN(dot)(dg[i], hg[i]);
    REAL av = restvolume < 0 ? -restvolume : restvolume;
    if (av < (REAL)1.0e-20) av = (REAL)1.0e-20;
    REAL dt = X->dt;
    REAL dalpha = (REAL)1 / (mu * av * dt * dt);
    REAL halpha = (REAL)1 / (lam * av * dt * dt);
    REAL ddamp = 0, dgam = 1, hdamp = 0, hgam = 1;
    if (kd > (REAL)0) {
        REAL dbeta = mu * av * kd * dt * dt, hbeta = lam * av * kd * dt * dt;
        dgam = dalpha * dbeta / dt;
        hgam = halpha * hbeta / dt;
        for (int i = 0; i < 4; ++i) {
            VEC dv = FN(sub)(P[i], FN(ld)(X->pprev, p[i]));
            ddamp += FN(dot)(dg[i], dv);
            hdamp += FN(dot)(hg[i], dv);
        }
        ddamp = ddamp * dgam;
        hdamp = hdamp * hgam;
        dgam = dgam + (REAL)1;
        hgam = hgam + (REAL)1;
    }
    REAL Axx = dgam * dsw + dalpha, Ayy = hgam * hsw + halpha;
    REAL detA = Axx * Ayy - dh * dh;
    if (detA < (REAL)1.0e-8) return 0;
    REAL invd = (REAL)1 / detA;
    REAL db = -dC - dalpha * (REAL)0 - ddamp;
    REAL hb = -hC - halpha * (REAL)0 - hdamp;
    REAL ddL = invd * (Ayy * db - dh * hb);
    REAL hdL = invd * (Axx * hb - dh * db);
    for (int i = 0; i < 4; ++i) {
        VEC dv = FN(scl)(im[i], FN(add)(FN(scl)(ddL, dg[i]), FN(scl)(hdL, hg[i])));
        out[i][0] = dv.x; out[i][1] = dv.y; out[i][2] = dv.z;
    }
    return 0xF;
}

static int FN(con_attach)(const FN(ctx) * X, int c, REAL out[4][3]) {
    REAL k = X->c_stiffness[c];
    if (k <= (REAL)0) return 0;
    int pt1 = X->c_pts[4 * c];
    VEC tgt = FN(mk)(X->c_restvector[4 * c], X->c_restvector[4 * c + 1], X->c_restvector[4 * c + 2]);
    REAL im1 = FN(invm)(X->mass, X->stopped, pt1);
    if (im1 == (REAL)0) return 0;
    VEC p1 = FN(ld)(X->pos, pt1);
    VEC n = FN(sub)(p1, tgt);
    REAL d = FN(len)(n);
    if (!(d >= (REAL)1.0e-6)) return 0;
    REAL alpha = (REAL)1 / k;
    alpha = alpha / (X->dt * X->dt);
    REAL C = d - X->c_restlength[c];
    n = FN(dvs)(n, d);
    REAL dsum = 0, gamma = 1;
    REAL kd = X->c_damp[c];
    if (kd > (REAL)0) {
        VEC pv = FN(ld)(X->pprev, pt1);
        REAL beta = k * kd * X->dt * X->dt;
        gamma = alpha * beta / X->dt;
        dsum = gamma * FN(dot)(n, FN(sub)(p1, pv));
        gamma = gamma + (REAL)1;
    }
    REAL dL = (-C - alpha * (REAL)0 - dsum) / (gamma * im1 + alpha);
    VEC dp = FN(scl)(-dL, n);
    VEC dd = FN(scl)(-im1, dp);
    out[0][0] = dd.x; out[0][1] = dd.y; out[0][2] = dd.z;
    return 0x1;
}

/* Vertex->constraint-slot CSR in table order (built once per table). */
long FN(orc_csr_size)(int ncons, const int* c_type, const int* c_pts) {
    long n = 0;
    for (int c = 0; c < ncons; ++c) n += (c_type[c] == T_ATTACH) ? 1 : 4;
    (void)c_pts;
    return n;
}
void FN(orc_build_csr)(int nv, int ncons, const int* c_type, const int* c_pts, long* row, long* slot) {
    for (int v = 0; v <= nv; ++v) row[v] = 0;
    for (int c = 0; c < ncons; ++c) {
        int k = (c_type[c] == T_ATTACH) ? 1 : 4;
        for (int i = 0; i < k; ++i) row[c_pts[4 * c + i] + 1]++;
    }
    for (int v = 0; v < nv; ++v) row[v + 1] += row[v];
    long* fill = (long*)malloc(sizeof(long) * (size_t)(nv + 1));
    for (int v = 0; v <= nv; ++v) fill[v] = row[v];
    for (int c = 0; c < ncons; ++c) {
        int k = (c_type[c] == T_ATTACH) ? 1 : 4;
        for (int i = 0; i < k; ++i) slot[fill[c_pts[4 * c + i]]++] = 4L * c + i;
    }
    free(fill);
}

/* One Jacobi projection of the whole table (solve_constraints with
 * use_jacobi=1, engine.py:1029-1052 -> _dispatch_constraints :890-1027) into
 * dP/dPw, which are overwritten (clear() + accumulate).  Supported types:
 * TETARAPSVD, TETVOLUME, TETARAPANISO, TETSNH, ATTACH; other types are
 * skipped.  corr is scratch of 12*ncons REAL, mask of ncons int. */
void FN(orc_project)(int nv, const REAL* pos, const REAL* pprev, const REAL* mass, const int* stopped,
                     const REAL* rest_matrix, const REAL* v_fiber, const REAL* activation, const REAL* tendonmask,
                     int ncons, const int* c_type, const int* c_pts, const REAL* c_stiffness, const REAL* c_damp,
                     const int* c_tetid, const REAL* c_restlength, const REAL* c_restvector, const REAL* c_restdir,
                     REAL dt, REAL contraction_ratio, REAL fiber_stiffness_scale,
                     const long* csr_row, const long* csr_slot, REAL* corr, int* mask,
                     REAL* dP, REAL* dPw) {
    FN(ctx) X;
    X.nv = nv; X.pos = pos; X.pprev = pprev; X.mass = mass; X.stopped = stopped;
    X.rest_matrix = rest_matrix; X.v_fiber = v_fiber; X.activation = activation; X.tendonmask = tendonmask;
    X.c_type = c_type; X.c_pts = c_pts; X.c_stiffness = c_stiffness; X.c_damp = c_damp; X.c_tetid = c_tetid;
    X.c_restlength = c_restlength; X.c_restvector = c_restvector; X.c_restdir = c_restdir;
    X.dt = dt; X.contraction_ratio = contraction_ratio; X.fiber_stiffness_scale = fiber_stiffness_scale;
#pragma omp parallel for schedule(dynamic, 1024)
    for (int c = 0; c < ncons; ++c) {
        REAL out[4][3];
        int m = 0;
        switch (c_type[c]) {
            case T_TETARAPSVD: m = FN(con_arapsvd)(&X, c, out); break;
            case T_TETVOLUME: m = FN(con_volume)(&X, c, out); break;
            case T_TETARAPANISO: m = FN(con_aniso)(&X, c, out); break;
            case T_TETSNH: m = FN(con_snh)(&X, c, out); break;
            case T_ATTACH: m = FN(con_attach)(&X, c, out); break;
            default: m = 0;
        }
        mask[c] = m;
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 3; ++j) corr[12L * c + 3 * i + j] = (m >> i & 1) ? out[i][j] : (REAL)0;
    }
#pragma omp parallel for schedule(static)
    for (int v = 0; v < nv; ++v) {
        REAL sx = 0, sy = 0, sz = 0, w = 0;
        for (long e = csr_row[v]; e < csr_row[v + 1]; ++e) {
            long s = csr_slot[e];
            long c = s >> 2;
            int i = (int)(s & 3);
            if (mask[c] >> i & 1) {
                sx += corr[12 * c + 3 * i];
                sy += corr[12 * c + 3 * i + 1];
                sz += corr[12 * c + 3 * i + 2];
                w += (REAL)1;
            }
        }
        dP[3L * v] = sx; dP[3L * v + 1] = sy; dP[3L * v + 2] = sz;
        dPw[v] = w;
    }
}

/* ------------------------------------------------------------------------ */
/* Metrics. count_inverted_tets_kernel engine.py:410-428; calc_vol_error_kernel
 * engine.py:701-718; arap_residual_accum_kernel mg/kernel.py:86-117. */
int FN(orc_count_inverted)(int nt, const int* tets, const REAL* pos, const REAL* rest_matrix) {
    int n = 0;
    for (int c = 0; c < nt; ++c) {
        const int* p = tets + 4 * c;
        VEC p3 = FN(ld)(pos, p[3]);
        MAT F = FN(mul)(FN(cols)(FN(sub)(FN(ld)(pos, p[0]), p3), FN(sub)(FN(ld)(pos, p[1]), p3), FN(sub)(FN(ld)(pos, p[2]), p3)),
                        FN(ldB)(rest_matrix, c));
        if (FN(det)(F) <= (REAL)0) ++n;
    }
    return n;
}
double FN(orc_total_volume)(int nt, const int* tets, const REAL* pos) {
    double acc = 0;
    for (int c = 0; c < nt; ++c) {
        const int* p = tets + 4 * c;
        VEC p0 = FN(ld)(pos, p[0]);
        VEC d1 = FN(sub)(FN(ld)(pos, p[1]), p0), d2 = FN(sub)(FN(ld)(pos, p[2]), p0), d3 = FN(sub)(FN(ld)(pos, p[3]), p0);
        acc += (double)(FN(dot)(FN(cross)(d2, d1), d3) / (REAL)6);
    }
    return acc;
}
/* Per-tet ARAP-SVD constraint value C=||sigma-1|| (the residual whose max and
 * RMS the parity gate compares). */
void FN(orc_arap_residual)(int nt, const int* tets, const REAL* pos, const REAL* rest_matrix, REAL* C_out) {
#pragma omp parallel for schedule(static)
    for (int c = 0; c < nt; ++c) {
        const int* p = tets + 4 * c;
        VEC p3 = FN(ld)(pos, p[3]);
        MAT F = FN(mul)(FN(cols)(FN(sub)(FN(ld)(pos, p[0]), p3), FN(sub)(FN(ld)(pos, p[1]), p3), FN(sub)(FN(ld)(pos, p[2]), p3)),
                        FN(ldB)(rest_matrix, c));
        MAT U, V; VEC s;
        FN(svdm)(F, &U, &s, &V);
        REAL a = s.x - 1, b = s.y - 1, d = s.z - 1;
        C_out[c] = SQRT(a * a + b * b + d * d);
    }
}


/* ------------------------------------------------------------------------ */
/* Bone push-out on a grid SDF.  The reference queries the bone triangle mesh
 * (solve_mesh_contact_pos_kernel, sdf/kernel.py:122-170): err = dist - offset;
 * if err < 0 (and -err <= max_push when max_push > 0) pos -= n * err, n the
 * outward normal; inverse-mass-0 vertices are skipped.  With capsule bones the
 * distance comes from the baked grid: trilinear phi, n = normalised analytic
 * gradient of the trilinear interpolant. */
static REAL FN(cap_phi)(const REAL* a, const REAL* b, REAL r, const REAL* x) {
    REAL ab[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]}, ax[3] = {x[0] - a[0], x[1] - a[1], x[2] - a[2]};
    REAL L2 = ab[0] * ab[0] + ab[1] * ab[1] + ab[2] * ab[2];
    REAL t = 0;
    if (L2 > 0) {
        t = (ax[0] * ab[0] + ax[1] * ab[1] + ax[2] * ab[2]) / L2;
        t = t < 0 ? 0 : (t > 1 ? 1 : t);
    }
    REAL d[3] = {ax[0] - t * ab[0], ax[1] - t * ab[1], ax[2] - t * ab[2]};
    return SQRT(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) - r;
}

/* caps: [n][8] = center xyz, half, axis xyz, radius; transforms [n][12] or NULL. */
void FN(orc_sdf_bake_capsules)(int nx, int ny, int nz, const REAL* origin, REAL h, int ncaps, const REAL* caps,
                               const REAL* transforms, REAL band, REAL* phi) {
    REAL* seg = (REAL*)malloc(sizeof(REAL) * 7 * (size_t)(ncaps > 0 ? ncaps : 1));
    for (int c = 0; c < ncaps; ++c) {
        const REAL* K = caps + 8 * c;
        REAL a[3], b[3];
        for (int k = 0; k < 3; ++k) {
            a[k] = K[k] - K[3] * K[4 + k];
            b[k] = K[k] + K[3] * K[4 + k];
        }
        if (transforms) {
            const REAL* T = transforms + 12 * c;
            REAL a0[3] = {a[0], a[1], a[2]}, b0[3] = {b[0], b[1], b[2]};
            for (int r = 0; r < 3; ++r) {
                a[r] = T[4 * r] * a0[0] + T[4 * r + 1] * a0[1] + T[4 * r + 2] * a0[2] + T[4 * r + 3];
                b[r] = T[4 * r] * b0[0] + T[4 * r + 1] * b0[1] + T[4 * r + 2] * b0[2] + T[4 * r + 3];
            }
        }
        for (int k = 0; k < 3; ++k) { seg[7 * c + k] = a[k]; seg[7 * c + 3 + k] = b[k]; }
        seg[7 * c + 6] = K[7];
    }
#pragma omp parallel for schedule(static)
    for (int iz = 0; iz < nz; ++iz)
        for (int iy = 0; iy < ny; ++iy)
            for (int ix = 0; ix < nx; ++ix) {
                REAL x[3] = {origin[0] + h * (REAL)ix, origin[1] + h * (REAL)iy, origin[2] + h * (REAL)iz};
                REAL v = band;
                for (int c = 0; c < ncaps; ++c) {
                    REAL pc = FN(cap_phi)(seg + 7 * c, seg + 7 * c + 3, seg[7 * c + 6], x);
                    if (pc < v) v = pc;
                }
                phi[((size_t)iz * ny + iy) * nx + ix] = v;
            }
    free(seg);
}

void FN(orc_sdf_push)(int nv, REAL* pos, const REAL* inv_mass, const REAL* phi, int nx, int ny, int nz,
                      const REAL* origin, REAL h, REAL offset, REAL max_push) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nv; ++i) {
        if (inv_mass[i] == (REAL)0) continue;
        REAL inv_h = (REAL)1 / h;
        REAL gx = (pos[3 * i] - origin[0]) * inv_h, gy = (pos[3 * i + 1] - origin[1]) * inv_h,
             gz = (pos[3 * i + 2] - origin[2]) * inv_h;
        if (!(gx >= 0 && gy >= 0 && gz >= 0 && gx <= (REAL)(nx - 1) && gy <= (REAL)(ny - 1) && gz <= (REAL)(nz - 1)))
            continue;
        int ix = (int)gx, iy = (int)gy, iz = (int)gz;
        if (ix > nx - 2) ix = nx - 2;
        if (iy > ny - 2) iy = ny - 2;
        if (iz > nz - 2) iz = nz - 2;
        REAL fx = gx - (REAL)ix, fy = gy - (REAL)iy, fz = gz - (REAL)iz;
        size_t sy = (size_t)nx, sz = (size_t)nx * ny;
        const REAL* b = phi + iz * sz + iy * sy + ix;
        REAL c000 = b[0], c100 = b[1], c010 = b[sy], c110 = b[sy + 1];
        REAL c001 = b[sz], c101 = b[sz + 1], c011 = b[sz + sy], c111 = b[sz + sy + 1];
        REAL c00 = c000 + fx * (c100 - c000), c10 = c010 + fx * (c110 - c010);
        REAL c01 = c001 + fx * (c101 - c001), c11 = c011 + fx * (c111 - c011);
        REAL c0 = c00 + fy * (c10 - c00), c1 = c01 + fy * (c11 - c01);
        REAL ph = c0 + fz * (c1 - c0);
        REAL dx0 = (c100 - c000) + fy * ((c110 - c010) - (c100 - c000));
        REAL dx1 = (c101 - c001) + fy * ((c111 - c011) - (c101 - c001));
        REAL dy0 = (c010 - c000) + fx * ((c110 - c100) - (c010 - c000));
        REAL dy1 = (c011 - c001) + fx * ((c111 - c101) - (c011 - c001));
        REAL g[3] = {(dx0 + fz * (dx1 - dx0)) * inv_h, (dy0 + fz * (dy1 - dy0)) * inv_h, (c1 - c0) * inv_h};
        REAL gl = SQRT(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
        if (!(gl > (REAL)1e-12)) continue;
        REAL err = ph - offset;
        if (err < 0 && (max_push <= 0 || -err <= max_push)) {
            for (int k = 0; k < 3; ++k) pos[3 * i + k] -= (g[k] / gl) * err;
        }
    }
}

#undef VEC
#undef MAT
#undef SQRT
#undef T_ATTACH
#undef T_TETVOLUME
#undef T_TETARAPSVD
#undef T_TETARAPANISO
#undef T_TETSNH
