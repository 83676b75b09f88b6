/*
 * xpbd_b200.h -- C ABI of libxpbd_b200.so, the sm_100a XPBD substep.
 *
 * Every buffer is a device pointer owned by the caller (the library never
 * allocates on these entry points).  Arrays documented as [n][4] hold four
 * floats per element and must be 16-byte aligned.  All launches go to the
 * given stream; no entry point synchronises, so every call may be captured
 * into a CUDA graph.  Return value: XPBD_OK or a negative XPBD_ERR_* code
 * (xpbd_error_string() describes the last failure on the calling thread).
 *
 * Each entry point names the reference (chunleili/rlmuscleV2) code it
 * replaces.  The reference launches one Warp kernel per constraint type per
 * iteration and scatters with float atomics into dP/dPw; this library keeps
 * the same arithmetic but projects all constraints of a tet in one pass over
 * Morton-ordered tiles (see XpbdTiles).
 */
#ifndef XPBD_B200_H
#define XPBD_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef void* xpbd_stream_t; /* a cudaStream_t */

enum {
    XPBD_OK = 0,
    XPBD_ERR_ARG = -1,    /* null pointer / bad size / bad enum */
    XPBD_ERR_ALIGN = -2,  /* a [n][4] array is not 16-byte aligned */
    XPBD_ERR_CUDA = -3,   /* a CUDA runtime call failed */
    XPBD_ERR_LIMIT = -4,  /* a size exceeds a documented maximum */
};

/* Device status word bits (OR-ed by kernels; the host reads and clears it). */
enum {
    XPBD_STATUS_PAIR_OVERFLOW = 1 << 0,    /* more candidate pairs than max_pairs (extra pairs dropped) */
    XPBD_STATUS_CONTACT_OVERFLOW = 1 << 1, /* more contacts than max_contacts (extra contacts dropped) */
    XPBD_STATUS_STACK_OVERFLOW = 1 << 2,   /* BVH traversal deeper than its stack (query cut short) */
    XPBD_STATUS_BARRIER_TIMEOUT = 1 << 3,  /* a grid-wide wait of the persistent pass gave up (results invalid) */
    XPBD_STATUS_MMA_TIMEOUT = 1 << 4,      /* a tensor-core GEMM gave up waiting for its MMAs (results invalid) */
    XPBD_STATUS_ACC_RANGE = 1 << 5,        /* a tet correction left the fixed-point accumulator's safe range */
};

#define XPBD_MAX_MATERIALS 64
#define XPBD_MAX_ATTACH_MATERIALS 16
#define XPBD_MAX_TILE_VERTS 4096

/* Material flags: which constraints a tet carries (constraint types of
 * src/muscle/defs.py:20-36). */
enum {
    XPBD_MAT_ARAPSVD = 1 << 0, /* TETARAPSVD   solve_kernels.py:1194 */
    XPBD_MAT_VOLUME = 1 << 1,  /* TETVOLUME    solve_kernels.py:553  */
    XPBD_MAT_ANISO = 1 << 2,   /* TETARAPANISO solve_kernels.py:1310 */
    XPBD_MAT_SNH = 1 << 3,     /* TETSNH       solve_kernels.py:1587 */
    XPBD_MAT_DAMPED = 1 << 4,  /* a constraint of this material reads pprev */
};

typedef struct XpbdMaterial {
    uint32_t flags;
    float arap_k;             /* TETARAPSVD stiffness (c_stiffness) */
    float vol_k, vol_damp;    /* TETVOLUME stiffness, dampingratio */
    float aniso_k;            /* TETARAPANISO stiffness */
    float snh_mu, snh_lam;    /* TETSNH c_stiffness, c_restdir[0] */
    float snh_damp;           /* TETSNH dampingratio */
} XpbdMaterial;

typedef struct XpbdAttachMaterial {
    float k;    /* ATTACH stiffness */
    float damp; /* ATTACH dampingratio */
} XpbdAttachMaterial;

typedef struct XpbdParams {
    float dt;                    /* substep dt */
    float gravity[3];            /* gravity vector (engine.py:799-803) */
    float veldamping;            /* integrate_kernel velocity damping */
    int32_t quasi_static;        /* integrate_kernel quasi_static */
    float omega;                 /* Jacobi relaxation of the averaged correction; 1 = reference */
    float contraction_ratio;     /* aniso_arap activation scale */
    float fiber_stiffness_scale; /* aniso_arap stiffness multiplier */
    int32_t n_materials;
    int32_t n_attach_materials;
    int32_t tile_variant;        /* bit 0: flip the tile pass's CTAs/SM (default 3 at 80 regs for the
                                    ARAP/aniso set, 2 at up to 128 regs with volume/SNH/damping);
                                    bit 1: ARAP-SVD through the SVD even where the polar rotation applies;
                                    bit 2: persistent pass loads the next tet's streams ahead (prefetch);
                                    bit 3: undamped light and volume sets two tets per thread on packed
                                    FP32x2 arithmetic (slower on B200: the register pairing costs as
                                    many moves as it saves FP32 instructions);
                                    bit 4: persistent pass keeps the runtime shared-memory layout for
                                    tiles of <= 768 vertices (default: compile-time offsets);
                                    bit 5: the per-iteration tile pass asks the copy engine for an L2
                                    prefetch of its tile's tet streams (cp.async.bulk.prefetch.L2)
                                    before staging the tile's vertices;
                                    bit 6: tets whose ARAP rotation needs the SVD (det F <= 1e-6 |F|^3)
                                    are projected in a deferred pass of the whole CTA after the tile's
                                    loop instead of where the loop meets them (same results bit for
                                    bit; pays where such tets are common) */
    float acc_scale;             /* > 0: the tile passes sum each tet's corrections into shared memory as
                                    32-bit integers round(d * acc_scale) (native integer atomics; shared
                                    float atomics cost ~5x more) and read the sums back as float(sum) /
                                    acc_scale; xpbd_acc_scale_for_extent gives the value for a mesh */
    float arap_skip_ssq;         /* ARAP-SVD leaves a tet out (no correction, not counted in the Jacobi
                                    divisor) when sum((sigma-1)^2) is below a threshold: 0 selects the
                                    reference's 1e-12 (solve_kernels.py:1257-1259), > 0 that value, < 0
                                    no threshold (only an exact rotation is left out).  Whether a
                                    near-rest tet passes 1e-12 is decided by FP32 rounding; parity tests
                                    disable it to compare everything else at rounding level */
    int32_t* status;             /* optional [1]: XPBD_STATUS_ACC_RANGE is or-ed in when the sum of a single
                                    tet's 12 correction magnitudes exceeds 1/64 of the fixed-point range, or
                                    is NaN or Inf (a vertex sum can then wrap only with > 64 such tets) */
    XpbdMaterial materials[XPBD_MAX_MATERIALS];
    XpbdAttachMaterial attach[XPBD_MAX_ATTACH_MATERIALS];
} XpbdParams;

/* Per-vertex state, in the library's (tile-grouped Morton) vertex order. */
typedef struct XpbdVerts {
    int32_t n;
    int32_t reserved;
    float* pos;                 /* [n][4] x, y, z, inverse mass (0 = stopped/massless) */
    float* pprev;               /* [n][4] x, y, z, unused */
    float* vel;                 /* [n][4] vx, vy, vz, stopped flag (0/1) */
    const float* mass;          /* [n] lumped mass */
    const float* force;         /* [n][4] external force or NULL */
    float* accum;               /* [n][4] Jacobi accumulator dP.xyz, dPw; zero between iterations */
    const int32_t* vflags;      /* [n] or NULL: bits 0-7 attach material+1 (0 = none), bit 8 pin */
    const float* attach_target; /* [n][4] x, y, z, restlength (ATTACH c_restvector / c_restlength) */
    const float* pin_target;    /* [n][4] x, y, z, active (target_pos + rest_offset, pin_active) */
} XpbdVerts;

#define XPBD_VF_ATTACH_MASK 0xff
#define XPBD_VF_PIN (1 << 8)

/* Morton tiles of tets.  Tile t owns tets [tile_tptr[t], tile_tptr[t+1]) and
 * the vertex list tile_verts[tile_vptr[t] .. tile_vptr[t+1]); the first
 * tile_nint[t] of those are interior (touched by no other tile), the rest
 * are tile-boundary vertices.  tet_q[t] = {l0 | l1<<16, l2 | l3<<16,
 * material, bits of the signed rest volume V0}, l* being tile-local vertex
 * indices (reference order pts[0..3], pts[3] the rest-matrix reference
 * vertex).  The rest matrix B = inv(Dm) is row-major over
 * tet_b0 = {B00,B01,B02,B10}, tet_b1 = {B11,B12,B20,B21}, tet_b2 = {B22}. */
typedef struct XpbdTiles {
    int32_t n_tets, n_tiles, n_boundary, max_tile_verts;
    const int32_t* tile_vptr;  /* [n_tiles+1] */
    const int32_t* tile_nint;  /* [n_tiles] */
    const int32_t* tile_tptr;  /* [n_tiles+1] */
    const int32_t* tile_verts; /* [tile_vptr[n_tiles]] global vertex ids */
    const uint32_t* tet_q;     /* [n_tets][4] */
    const float* tet_b0;       /* [n_tets][4] */
    const float* tet_b1;       /* [n_tets][4] */
    const float* tet_b2;       /* [n_tets] */
    const float* tet_fiber;    /* [n_tets][4] f0.xyz, tendonmask; NULL without aniso */
    const float* tet_act;      /* [n_tets] activation; NULL without aniso */
    const int32_t* bnd_verts;  /* [n_boundary] boundary vertex ids */
    const int32_t* vert_ntiles; /* [n_verts] number of tiles touching each vertex (FUSED_LAST mode) */
    int32_t* arrive;            /* [n_verts] arrival counters, zero between iterations (FUSED_LAST mode) */
} XpbdTiles;

/* Grid signed-distance field of the bones, phi[z][y][x], x fastest. */
typedef struct XpbdSdf {
    const float* phi;
    int32_t nx, ny, nz;
    float origin[3];
    float h;               /* cell size (grid node spacing) */
    float contact_offset;  /* push out until phi >= contact_offset */
    float max_push;        /* > 0: ignore contacts deeper than this; <= 0: push all */
    int32_t reserved;
} XpbdSdf;

typedef struct XpbdMetrics {
    double vol_sum;        /* sum of signed tet volumes (calc_vol_error_kernel, engine.py:701) */
    double resid_sq_sum;   /* sum of ARAP C^2 (arap_residual_accum_kernel, mg/kernel.py:86) */
    float resid_max;       /* max ARAP C = ||sigma - 1|| */
    int32_t n_inverted;    /* tets with det F <= 0 (count_inverted_tets_kernel, engine.py:410) */
    int32_t n_nonfinite;   /* tets touching a non-finite position */
    int32_t reserved;
} XpbdMetrics;

/* vertex_step ops, applied in this order to each vertex. */
enum {
    XPBD_OP_SDF = 1 << 0,      /* bone push-out (solve_mesh_contact_pos_kernel, sdf/kernel.py:122-170) */
    XPBD_OP_VELOCITY = 1 << 1, /* update_velocities_kernel, engine.py:582-605 */
    XPBD_OP_PREDICT = 1 << 2,  /* integrate_kernel, engine.py:431-464 */
    XPBD_OP_PIN = 1 << 3,      /* pintotarget_overwrite_masked_kernel, mg/kernel.py:211-225 */
};

/* apply ops for xpbd_apply_all / xpbd_apply_boundary. */
enum {
    XPBD_APPLY_ATTACH = 1 << 0, /* add ATTACH corrections (solve_attach_kernel, solve_kernels.py:892) to accum */
    XPBD_APPLY_DIVIDE = 1 << 1, /* pos += omega * dP / dPw (apply_dP_kernel, engine.py:689-698) */
    XPBD_APPLY_PIN = 1 << 2,    /* pin overwrite (mg/kernel.py:211-225) */
    XPBD_APPLY_CLEAR = 1 << 3,  /* zero accum after reading (clear_dP_kernel, engine.py:664) */
};

/* project modes */
enum {
    XPBD_PROJECT_FUSED = 0,      /* apply interior vertices in place, accumulate boundary ones */
    XPBD_PROJECT_ACCUMULATE = 1, /* accumulate every vertex into accum (reference dP/dPw) */
    XPBD_PROJECT_FUSED_LAST = 2, /* FUSED, and the last tile to reach a boundary vertex finishes it:
                                    a whole Jacobi iteration in one launch (needs vert_ntiles, arrive) */
};

int xpbd_abi_version(void);

/* XpbdParams.acc_scale for the length max_coord: the largest power of two s
 * with s x max_coord <= 2^26.  One tet whose 12 correction magnitudes sum
 * above 2^25 / s (between max_coord / 2 and max_coord), or to NaN/Inf, sets
 * XPBD_STATUS_ACC_RANGE; a vertex's sum may reach 64 such tets before the
 * 32-bit range ends; the quantum is 1/s.  The engine passes 128 x the longest
 * rest edge of the mesh (a projection moves a sane tet's vertices by a few
 * edge lengths), which gives 1/s = 1.5e-8 m on a mesh of 5.5 mm edges.
 * Library-specific (the reference sums corrections with float atomics). */
float xpbd_acc_scale_for_extent(float max_coord);

const char* xpbd_error_string(void);

/* Fused per-vertex substep boundary: [push-out] -> [velocity] -> [predict] -> [pin].
 * Replaces XpbdEngine.integrate (engine.py:798-809), update_velocities
 * (engine.py:811-829), MultiGridSim.apply_pintotarget (mg/mg.py:1251-1261)
 * and the AnimatedBoneMeshCollider push-out (example/humanV2.py:400-406). */
int xpbd_vertex_step(const XpbdParams* prm, const XpbdVerts* v, uint32_t ops, const XpbdSdf* sdf,
                     xpbd_stream_t stream);

/* One Jacobi projection of every tet constraint.  Replaces
 * XpbdEngine.solve_constraints / _dispatch_constraints (engine.py:1029-1052,
 * 890-1027) and, in FUSED mode, apply_dP (engine.py:865) for interior
 * vertices. */
int xpbd_project(const XpbdParams* prm, const XpbdTiles* tiles, const XpbdVerts* v, int32_t mode,
                 xpbd_stream_t stream);

/* Finish a FUSED projection on the tile-boundary vertices: ATTACH, divide,
 * pin, clear (apply ops as above). */
int xpbd_apply_boundary(const XpbdParams* prm, const XpbdTiles* tiles, const XpbdVerts* v, uint32_t ops,
                        xpbd_stream_t stream);

/* Apply ops over every vertex (the unfused engine primitives: ATTACH
 * accumulation of solve_constraints, apply_dP, apply_pintotarget, clear). */
int xpbd_apply_all(const XpbdParams* prm, const XpbdVerts* v, uint32_t ops, xpbd_stream_t stream);

/* Masked hard pin in the reference's own layout: pos4[pts[i]].xyz =
 * target[i] + offset[i] where active[i] != 0 (target/offset are [n][3]).
 * pintotarget_overwrite_masked_kernel, mg/kernel.py:211-225. */
int xpbd_pin_overwrite_masked(int32_t n, const int32_t* pts, const float* target, const float* offset,
                              const int32_t* active, float* pos4, xpbd_stream_t stream);

/* SVD inversion repair, XpbdEngine.repair_inverted_tets (engine.py:831-856):
 * iters passes of (accumulate, apply).  Accumulate
 * (_svd_clamp_accumulate_kernel, engine.py:293-367): every tet whose
 * sign-fixed singular values of F = Ds B are not all >= sigma_min takes the
 * edge matrix U diag(max(s, sigma_min)) V^T inverse(B), its differences
 * d0..d2 from the current edges p_i - p3, shifted by (d0 + d1 + d2) / 4 so
 * the centroid stays (d3 = -shift), and adds them with a count of 1 to the
 * accumulator of each vertex that is not stopped (vel.w == 0).  Apply
 * (_apply_svd_clamp_kernel, engine.py:370-380): pos += alpha dP / w where
 * w > 0.  The accumulator is zeroed first and left zeroed; a no-op when
 * iters == 0 or alpha <= 0.  Sums use float atomics (order-dependent in
 * the last bits; the repair is off the hot pass). */
int xpbd_svd_clamp(const XpbdTiles* tiles, const XpbdVerts* v, float sigma_min, float alpha, int32_t iters,
                   xpbd_stream_t stream);

/* Mesh metrics into out (device XpbdMetrics, zeroed by this call). */
int xpbd_metrics(const XpbdTiles* tiles, const XpbdVerts* v, XpbdMetrics* out, xpbd_stream_t stream);

/* Per-frame kinematic targets of bone-bound vertices.  transforms is
 * [n_bones][12] = row-major 3x4 [R | t]; vertex i (library order) rides bones
 * vert_bone[i][0..1] with blend weight vert_w[i] (NULL = 0) from rest
 * position rest4[i] (x,y,z,-): target = (1-w)(R_a x + t_a) + w (R_b x + t_b)
 * (two-bone linear blend skinning, the reference's target_mode="lbs",
 * mg/mg.py:1176-1209), written to pin_target[i].xyz and
 * attach_target[i].xyz (their .w lanes are kept).  Replaces the per-frame
 * target refresh of MultiGridSim (load_frame_targets /
 * _update_belly_attach_targets, mg/mg.py:1386-1407, 725-734) without the
 * reference's device->host->device round trip. */
int xpbd_bone_targets(int32_t n, int32_t n_bones, const float* transforms, const int32_t* vert_bone,
                      const float* vert_w, const float* rest4, float* pin_target, float* attach_target,
                      xpbd_stream_t stream);

/* Soft pull toward per-vertex targets: for i < n, v = idx[i] (idx NULL: v = i,
 * n <= n_verts), pos4[v].xyz += beta (target4[v].xyz - pos4[v].xyz), one
 * fma per component; beta finite (1 snaps, < 1 follows partly); idx entries
 * outside [0, n_verts) are skipped.  Two reference kernels are this operation:
 * presubframe_pintotarget_kernel (mg/kernel.py:229-257; MultiGridSim
 * .apply_pintotarget_all, mg/mg.py:1386-1397: every constraint point blended
 * toward target_pos + rest_offset once per kinematic step, after the hard
 * pin) and dense_soft_attach_kernel (mg/kernel.py:64-84; the coarse cage's
 * Neumann attach after each coarse ARAP sweep, mg/mg.py:1047-1062, idx = the
 * coarse nodes with a nonzero restriction column). */
int xpbd_blend_to_target(int32_t n, const int32_t* idx, int32_t n_verts, float* pos4, const float* target4,
                         float beta, xpbd_stream_t stream);

/* Bone-surface binding, the reference's target_mode="mesh" driver.  A bone
 * surface is a triangle mesh: bone4 [n_bverts][4] (x, y, z, -), btris
 * [n_btris][3].  Barycentric (u, v) of face (A, B, C) weight A and B, C takes
 * 1 - u - v (Warp's mesh_eval_position); the face frame is t1 = unit(A - C),
 * n = unit((A - C) x (B - C)), t2 = n x t1 (_face_basis, mg/kernel.py:267-285).
 * The closest-point queries are a brute force over all faces (ties keep the
 * lowest face index), meant for bone surfaces of up to a few 10^4 faces.
 *
 * xpbd_bone_bind replaces bone_bind_kernel (mg/kernel.py:287-310): for each
 * query4[i] the closest face within max_dist, its (u, v) and the offset
 * R^T (query - closest point) in the face frame (face 0, zeros when none). */
int xpbd_bone_bind(int32_t n, const float* query4, int32_t n_bverts, const float* bone4, int32_t n_btris,
                   const int32_t* btris, float max_dist, int32_t* out_face, float* out_uv, float* out_local4,
                   xpbd_stream_t stream);

/* bone_slide_target_kernel (mg/kernel.py:313-347) on the current bone
 * surface: with reproject != 0 each vertex re-binds to its closest face of
 * muscle4 when that point lies within slide_range of its anchor (anchor_face,
 * anchor_uv: the bind at the start frame), updating bind_face, bind_uv and
 * local4; then target = closest point + R local, written to pin_target.xyz
 * and/or attach_target.xyz (either may be NULL; .w lanes kept).  Faces must
 * come from xpbd_bone_bind on a surface with the same triangles. */
int xpbd_bone_slide_targets(int32_t n, const float* muscle4, const int32_t* anchor_face, const float* anchor_uv,
                            int32_t* bind_face, float* bind_uv, float* local4, float slide_range, int32_t reproject,
                            float max_dist, int32_t n_bverts, const float* bone4, int32_t n_btris,
                            const int32_t* btris, float* pin_target, float* attach_target, xpbd_stream_t stream);

/* Rigid pose of bone-surface vertices for a frame: out4[j] = R_b rest4[j] + t_b,
 * b = vert_bone[j], transforms as for xpbd_bone_targets above ([n_bones][12]
 * row-major [R | t]).  Stands in for the per-frame bone-mesh upload of
 * MultiGridSim._update_slide_target (mg/mg.py:1160-1174) when the bones are
 * rigid (the synthetic capsule skeleton). */
int xpbd_bone_surface_pose(int32_t n_bverts, const float* rest4, const int32_t* vert_bone, int32_t n_bones,
                           const float* transforms, float* out4, xpbd_stream_t stream);

/* Fascia ride coupling (Fascia ride mode, fascia/fascia.py:442-522).
 * xpbd_surface_bind replaces fascia_bind_kernel (fascia.py:130-157): for each
 * query4[i] (fascia rest position) the closest face of the muscle surface
 * (surf4 [n_sverts][4], stris [n_stris][3]) within max_dist, its (u, v), the
 * signed normal gap (query - closest point) . n and ok = 1 (face 0, zeros and
 * ok = 0 when none); same barycentric convention, face normal and tie rule as
 * xpbd_bone_bind.  xpbd_surface_ride replaces fascia_ride_kernel
 * (fascia.py:160-176): fascia4[bound[i]].xyz <- position(face[i], uv[i]) on
 * the current surface + n * gap[i] (.w kept). */
int xpbd_surface_bind(int32_t n, const float* query4, int32_t n_sverts, const float* surf4, int32_t n_stris,
                      const int32_t* stris, float max_dist, int32_t* out_face, float* out_uv, float* out_gap,
                      int32_t* out_ok, xpbd_stream_t stream);
int xpbd_surface_ride(int32_t n_bound, const int32_t* bound, const int32_t* face, const float* uv, const float* gap,
                      const float* surf4, const int32_t* stris, float* fascia4, xpbd_stream_t stream);

/* Fascia squeeze mode (fascia/fascia.py:45-125, 524-566).  target4 is the
 * muscle's per-vertex bone target (the pin target: target + rest offset), in
 * the muscle library order.  xpbd_fascia_advect (fascia_advect_bone_kernel):
 * fascia4[i] += target4[follow[i]] - prev_world4[i], then prev_world4[i] =
 * target4[follow[i]] (once per frame).  xpbd_fascia_anchor
 * (fascia_anchor_bone_kernel): fascia4[local[i]].xyz = target4[cons[i]] +
 * offset4[i].  xpbd_fascia_glue (solve_glue_kernel): one-way XPBD distance
 * step per pair holding restlen[c], compliance[c] / dt^2, zero starting
 * multiplier, scaled by omega: only the muscle vertex moves (atomics), by its
 * inverse mass muscle4.w. */
int xpbd_fascia_advect(int32_t n, const int32_t* follow, const float* target4, float* prev_world4, float* fascia4,
                       xpbd_stream_t stream);
int xpbd_fascia_anchor(int32_t n, const int32_t* local, const int32_t* cons, const float* offset4,
                       const float* target4, float* fascia4, xpbd_stream_t stream);
int xpbd_fascia_glue(int32_t n, const int32_t* pair_fascia, const int32_t* pair_muscle, const float* restlen,
                     const float* compliance, const float* fascia4, float* muscle4, float dt, float omega,
                     xpbd_stream_t stream);

/* Muscle-to-muscle glue (solve_m2m_glue_kernel, mg/kernel.py:350-394; run by
 * MultiGridSim between apply_dP and apply_pintotarget, mg/mg.py:1346-1355):
 * one XPBD distance step per pair (pair_a[c], pair_b[c]) toward restlen[c]
 * with compliance[c] / dt^2 and a zero starting multiplier, scaled by omega,
 * added to both endpoints of pos4 (library order) with atomics.  Inverse
 * masses are pos4.w.  Pairs sharing a vertex update it concurrently, as the
 * reference's atomic version does. */
int xpbd_m2m_glue(int32_t n_pairs, const int32_t* pair_a, const int32_t* pair_b, const float* restlen,
                  const float* compliance, float* pos4, float dt, float omega, xpbd_stream_t stream);

/* Capsule bone, rest pose: centre, unit axis, half segment length, radius. */
typedef struct XpbdCapsule {
    float center[3];
    float half;
    float axis[3];
    float radius;
} XpbdCapsule;

/* Bake the grid SDF of the union of n capsules, each moved by its
 * transforms[bone] ([n][12], NULL = rest pose), into sdf->phi.  Values are
 * exact distances within band of a capsule surface and clamped to band
 * elsewhere (band > 0; push-out only reads phi near zero). */
int xpbd_sdf_bake_capsules(const XpbdSdf* sdf, int32_t n_caps, const XpbdCapsule* caps, const float* transforms,
                           float band, xpbd_stream_t stream);

/* Batched instances (config of many independent meshes packed in one vertex
 * set): one grid SDF per instance, all grids of nx*ny*nz nodes, grid i at
 * phi + i*nx*ny*nz with its own origin and cell size. */
typedef struct XpbdSdfBatch {
    const float* phi;         /* [n_inst][nz][ny][nx] */
    const float* frame;       /* [n_inst][4] origin xyz, cell size h */
    const int32_t* vert_inst; /* [n_verts] instance of each vertex (library order), < 0: no push-out */
    int32_t n_inst, nx, ny, nz;
    float contact_offset, max_push;
} XpbdSdfBatch;

/* Bake every instance's grid from its own caps_per_inst capsules
 * (caps[i*caps_per_inst ...], transforms [n_inst*caps_per_inst][12] or NULL),
 * as xpbd_sdf_bake_capsules does for one grid; one launch for all grids. */
int xpbd_sdf_bake_capsules_batched(const XpbdSdfBatch* sdf, int32_t caps_per_inst, const XpbdCapsule* caps,
                                   const float* transforms, float band, xpbd_stream_t stream);

/* xpbd_vertex_step with XPBD_OP_SDF reading each vertex's instance grid. */
int xpbd_vertex_step_batched(const XpbdParams* prm, const XpbdVerts* v, uint32_t ops, const XpbdSdfBatch* sdf,
                             xpbd_stream_t stream);

/* dst[i] = src[idx[i]] for float lanes of width `width` (1..4). */
int xpbd_gather(int32_t n, int32_t width, const int32_t* idx, const float* src, int32_t src_stride, float* dst,
                int32_t dst_stride, xpbd_stream_t stream);

/* Two-level multigrid transfer (hpbd V-cycle, mg/mg.py:1064-1079).  Coarse
 * vertex ids in the restriction/blocks are the cage's own ids (cage order);
 * coarse_lib maps them to the coarse engine's library order.  Fine ids are
 * fine library ids. */
typedef struct XpbdCage {
    int32_t n_fine, n_coarse, n_blocks, max_block;
    const int32_t* r_ptr;      /* [n_coarse+1] restriction CSR per coarse vertex (cage order) */
    const int32_t* r_fine;     /* [nnz] fine vertex */
    const float* r_w;          /* [nnz] prolongation weight of that fine vertex on this coarse vertex */
    const int32_t* blk_ptr;    /* [n_blocks+1] coarse vertices of block b: [blk_ptr[b], blk_ptr[b+1]) */
    const int32_t* blk_moff;   /* [n_blocks] offset of the block's dim x dim row-major (P^T P + lam I)^-1 in minv */
    const float* minv;
    const int32_t* coarse_lib; /* [n_coarse] cage order -> coarse library order */
    const int32_t* p_idx;      /* [n_fine][4] coarse library ids of the embedding tet, -1 = not embedded */
    const float* p_w;          /* [n_fine][4] barycentric weights (1-u-v-w, u, v, w) */
    float* resid;              /* [n_fine][4] scratch: fine residual x_f - P x_c(prior) */
    float* rhs;                /* [n_coarse][4] scratch: P^T resid per coarse vertex (cage order) */
} XpbdCage;

/* Regularised Galerkin restriction of the xyz lanes of fine4 into coarse4:
 * x_c = argmin |P x_c - x_f|^2 + lam |x_c - prior|^2 with prior = the current
 * contents of coarse4, computed as prior + (P^T P + lam I)^-1 P^T (x_f - P prior)
 * (restrict_galerkin_scatter_kernel + block_solve_kernel, mg/kernel.py:137-178,
 * with lam -> 0 the reference's operator; the CSR gather runs one warp per
 * coarse vertex, the block solve over row chunks of each block).  Optional: coarse_prev4 receives
 * the same values (the q_j snapshot, mg/mg.py:1077), and where
 * coarse_pin4[c].w != 0 the coarse position is then overwritten by
 * coarse_pin4[c].xyz (the coarse kinematic pin, mg/mg.py:1013-1026).  The
 * CSR gather runs one warp per coarse vertex, the block solve over 64-row
 * chunks of each block; no atomics. */
int xpbd_mg_restrict(const XpbdCage* cage, const float* fine4, float* coarse4, float* coarse_prev4,
                     const float* coarse_pin4, xpbd_stream_t stream);

/* Step 1 of the V-cycle without the Galerkin restriction (mg/mg.py:1006-1012,
 * mg_restrict_mode "galerkin" = the restricted bone target copied in, "none" =
 * the coarse keeps its own state; also after the coarse-in-fine readout of
 * mg_sync_restrict "c2f", mg/mg.py:992-996): over the cage's n_coarse vertices
 * (coarse library order) coarse4.xyz = src4.xyz when src4 is not NULL, then
 * coarse_prev4 (optional) receives coarse4 and the coarse kinematic pin
 * overwrites coarse4.xyz where coarse_pin4[c].w != 0, as xpbd_mg_restrict
 * does after its block solve.  src4 must not alias coarse4. */
int xpbd_mg_coarse_reset(const XpbdCage* cage, const float* src4, float* coarse4, float* coarse_prev4,
                         const float* coarse_pin4, xpbd_stream_t stream);

/* fine4.xyz += sum_k w_k (coarse4 - coarse_prev4)[p_idx_k] (prolong_delta_kernel,
 * mg/kernel.py:8-39), then the fine pin overwrite where vflags has
 * XPBD_VF_PIN and pin_target.w != 0 (vflags/pin_target may be NULL).  With
 * coarse_prev4 NULL the prolongation is absolute, fine4.xyz = sum_k w_k
 * coarse4[p_idx_k] (prolong_kernel, mg/kernel.py:181-203; mg_mode
 * "projection"), on the embedded vertices only.  Given a cage whose p_idx/p_w
 * embed the coarse vertices in fine tets (n_fine = the coarse vertex count,
 * p_idx = fine ids), the absolute form reads the coarse positions off the fine
 * mesh (restrict_c2f_kernel, mg/kernel.py:43-60; mg_sync_restrict "c2f"). */
int xpbd_mg_prolong_delta(const XpbdCage* cage, const float* coarse4, const float* coarse_prev4, float* fine4,
                          const int32_t* vflags, const float* pin_target, xpbd_stream_t stream);

/* Triangle-triangle DCD between surface triangles (UdcfDcdCollider,
 * collision/udcf/solver.py:146-457, BVH broadphase).  tris index vertices in
 * the library order of the pos4 buffer the calls receive; inverse mass is
 * read from pos4.w (0 = solid).  Scratch ws_* and the pair/contact buffers
 * are caller-owned; sizes from xpbd_dcd_workspace_query. */
typedef struct XpbdDcd {
    int32_t n_tris, n_verts, max_pairs, max_contacts;
    const int32_t* tris;      /* [n_tris][3] */
    const int32_t* tri_group; /* [n_tris] 0 movable, 1 static; NULL = all movable */
    int32_t allow_self;       /* movable-vs-movable pairs (UdcfParams.allow_self) */
    int32_t jacobi_avg;       /* 1: dP/count (UdcfParams.jacobi_avg), 0: summed dP */
    float thickness;          /* AABB padding (UdcfParams.thickness) */
    float offset_eps;         /* contact accept threshold (UdcfParams.offset, 1e-6) */
    float multiplier;         /* collisionConstraintMultiplier (1.01) */
    float friction_static, friction_dynamic;
    float max_push;           /* > 0: clamp contact depth (UdcfParams.max_push) */
    float box_lo[3], box_hi[3]; /* Morton quantisation box (centres outside are clamped) */
    int32_t* pairs;           /* [max_pairs][2] (i, j > i), deterministic order; 16-byte aligned */
    int32_t* n_pairs;         /* [1] candidate pairs found (may exceed max_pairs) */
    int32_t* n_contacts;      /* [1] contacts found (may exceed max_contacts) */
    int32_t* c_ids;           /* [max_contacts][8]: cur tri verts, pair index, closest tri verts, 0 */
    float* c_data;            /* [max_contacts][12]: n.xyz, C, b1.xyz, C1, b2.xyz, C2 */
    float* x_prev;            /* [n_verts][4] positions at the broadphase (friction reference) */
    float* dP;                /* [n_verts][4] response accumulator, zero between calls */
    int32_t* status;          /* [1] XPBD_STATUS_* bits */
    float* ws_nodes;          /* workspace: BVH node records (children's boxes) + leaf boxes */
    uint32_t* ws_keys;        /* [n_tris] Morton keys (sorted in place) */
    int32_t* ws_vals;         /* [n_tris] triangle ids in Morton order */
    uint32_t* ws_keys2;       /* [n_tris] sort ping-pong */
    int32_t* ws_vals2;        /* [n_tris] */
    int32_t* ws_hist;         /* radix histograms, scan scratch and the sort's four grid barrier words (its last
                                 four entries); zero before the first call */
    float* ws_bbox;           /* boxes of 32- and 1024-leaf Morton blocks (2 float4 each) */
    int32_t* ws_count;        /* [n_tris] pairs per Morton position, then their offsets */
    int32_t* ws_total;        /* [1] */
    int32_t* ws_slots;        /* [16][n_tris] first partners of each query (counting pass) */
    int32_t* ws_split;        /* [n_tris-1][4] leaf range and split of each internal node */
    int32_t refit_only;       /* 1: keep the Morton order and hierarchy of the last rebuild on this
                                 workspace and recompute the boxes only (same pair set; no sort, no
                                 split search).  Needs one earlier call with 0. */
} XpbdDcd;

/* Element counts of the DCD workspace arrays for n_tris triangles. */
typedef struct XpbdDcdWorkspaceSizes {
    int64_t nodes_floats, keys, hist, bbox_floats, count, slots, split;
} XpbdDcdWorkspaceSizes;

int xpbd_dcd_workspace_query(int32_t n_tris, XpbdDcdWorkspaceSizes* out);

/* AABBs, LBVH rebuild (Morton sort + Karras hierarchy + refit) and the
 * candidate pair list; snapshot_prev != 0 first copies pos4 to x_prev
 * (UdcfDcdCollider.solve with i_iter == 0, udcf/solver.py:365-382). */
int xpbd_dcd_broadphase(const XpbdDcd* dcd, const float* pos4, int32_t snapshot_prev, xpbd_stream_t stream);

/* Narrowphase on the pair list, response and Jacobi apply onto pos4
 * (narrow_kernel, respond_kernel, apply_kernel; udcf/kernel.py:316-474,
 * 713-822). */
int xpbd_dcd_narrow_respond(const XpbdDcd* dcd, float* pos4, xpbd_stream_t stream);

/* Allocation-free Jacobi iteration.  This entry point has no counterpart in
 * the reference.  It is for callers that cannot allocate device memory or
 * hand the library a scratch buffer: a step recorded inside another
 * framework's CUDA graph capture (cudaMalloc is illegal during capture), a
 * plugin in a process whose GPU memory is owned by another allocator, a
 * real-time loop that forbids allocation after start-up.  It performs the
 * same fused iteration as xpbd_project(XPBD_PROJECT_FUSED) followed by
 * xpbd_apply_boundary(ATTACH | DIVIDE | PIN | CLEAR); v->accum is ignored and
 * the accumulator is instead a fixed device array of XPBD_NOALLOC_MAX_VERTS
 * float4 (4 MiB) that every GPU loading the library holds until process
 * exit.  Meshes with more than XPBD_NOALLOC_MAX_VERTS vertices are rejected
 * with XPBD_ERR_LIMIT.  Every call made outside stream capture looks up that
 * array's address (cudaGetSymbolAddress) on the current device; a call made
 * during capture reuses the last one found there, so the first call on a
 * device, and the first after a device reset, must come before any stream
 * capture (otherwise XPBD_ERR_ARG).  The array starts zeroed and each call
 * leaves it zeroed; it is cleared again only after a call that failed between
 * its two launches.  All calls share the array: calls that overlap on the GPU
 * race. */
#define XPBD_NOALLOC_MAX_VERTS 262144
int xpbd_iterate_noalloc(const XpbdParams* prm, const XpbdTiles* tiles, const XpbdVerts* v, xpbd_stream_t stream);

/* Persistent multi-iteration tet pass: state of xpbd_iterate_persistent. */
typedef struct XpbdPersist {
    const int32_t* tile_own; /* [n_tiles+1] tile k owns vertex ids [tile_own[k], tile_own[k+1]) (the vertices it
                                touches first); ids from tile_own[n_tiles] up to n_verts are in no tet */
    float* ring;             /* [3][n_verts][4] boundary accumulators; all zero before the first call */
    uint32_t* sync;          /* [4] two grid barrier counters, ring phase, counter parity; zero before the first call */
    int32_t* status;         /* [1] XPBD_STATUS_BARRIER_TIMEOUT; after it, zero ring and sync before the next call */
    int32_t tile_begin, tile_end; /* tiles [tile_begin, tile_end) in this launch (0, 0: all).  A sub-range must
                                     be closed (no vertex shared with tiles outside it, e.g. whole instances of a
                                     batch) and keeps its own sync words; vertices in no tet are finished by the
                                     launch whose range ends at n_tiles */
    /* Optional neighbour synchronisation (all three set, or all NULL for the grid-wide
     * barrier): tile t shares boundary vertices with tiles nbr_idx[nbr_ptr[t] ..
     * nbr_ptr[t+1]) (all inside the launched range); after its boundary sums a tile
     * publishes its iteration count in tile_cnt[t] and waits only until those
     * neighbours have published theirs, instead of waiting for every tile.  tile_cnt
     * holds one counter per tile, all zero before the first call and all equal between
     * calls (zero them with the ring and sync words after a barrier timeout). */
    const int32_t* nbr_ptr;  /* [n_tiles+1] */
    const int32_t* nbr_idx;  /* [nbr_ptr[n_tiles]] */
    uint32_t* tile_cnt;      /* [n_tiles] */
} XpbdPersist;

/* n_iters fused Jacobi iterations in ONE cooperative launch: the same
 * per-iteration result as n_iters x (xpbd_project(XPBD_PROJECT_FUSED) +
 * xpbd_apply_boundary(ATTACH | DIVIDE | PIN | CLEAR)), i.e. n_iters rounds of
 * solve_constraints -> apply_dP -> apply_pintotarget of MultiGridSim's
 * iteration phase (mg.py:1350-1360) with no hook in between.  Every tile's
 * vertices stay in shared memory for all iterations; tile-boundary sums go
 * through a ring of three global accumulators with one grid-wide barrier per
 * iteration, and pos is written once at the end.  Needs all n_tiles CTAs
 * resident at once (xpbd_persistent_fits); returns XPBD_ERR_LIMIT otherwise.
 * Barrier waits are bounded (about a second); on timeout the status bit is
 * set and the kernel runs to its end, every later barrier giving up within
 * 64 polls.  At most 2^20 iterations per call. */
int xpbd_iterate_persistent(const XpbdParams* prm, const XpbdTiles* tiles, const XpbdVerts* v,
                            const XpbdPersist* ps, int32_t n_iters, xpbd_stream_t stream);
/* *fits = 1 when the persistent pass of these materials can hold all tiles
 * resident on the current device; *slots (optional) = how many CTAs of it
 * can be resident at once (the largest tile range one launch can take). */
int xpbd_persistent_fits(const XpbdParams* prm, const XpbdTiles* tiles, int32_t* fits, int32_t* slots);

/* ---- Learned coarse correction: the per-cage-vertex MLP's kernels.  These
 * have no counterpart in the reference (its solver has no learned part); they
 * serve the learned warm start of the cage (forward, backward, Adam). ---- */

/* C[m][n] = sum_k A[m][k] B[n][k] on the tensor cores (tcgen05, BF16 operands,
 * FP32 accumulation), then per element of C: z = C + bias[n] (bias optional);
 * z *= gelu'(gelu_grad_of[m][n]) (optional, backward through a GELU whose
 * pre-activation is stored there); out_pre = z; y = act ? gelu(z) : z
 * (GELU tanh form of Hendrycks & Gimpel); out_f32 = y; out_bf16 = bf16(y);
 * out_bf16_t[n][m] = bf16(y) (every output optional).  A and B are BF16
 * row-major along k; k % 64 == 0; lda, ldb multiples of 8; rows of A beyond m
 * and of B beyond n read as zero. */
typedef struct XpbdGemm {
    const uint16_t* a;
    const uint16_t* b;
    int32_t lda, ldb, m, n, k, act;
    const float* bias;
    const float* gelu_grad_of;
    int32_t ld_g, ld_pre, ld_f32, ld_bf16, ld_bf16_t;
    int32_t flags;   /* XPBD_GEMM_THREAD_STAGED: operands staged by the CTA's threads instead of TMA */
    float* out_pre;
    float* out_f32;
    uint16_t* out_bf16;
    uint16_t* out_bf16_t;
    int32_t* status; /* XPBD_STATUS_MMA_TIMEOUT, optional */
} XpbdGemm;

#define XPBD_GEMM_THREAD_STAGED 1

/* One CTA per 128 x n_tile block of C (n_tile a multiple of 16, <= 256).  The
 * operands come into shared memory through the tensor memory accelerator
 * (cp.async.bulk.tensor 2-D boxes, up to four 64-wide k blocks in flight),
 * unless flags has XPBD_GEMM_THREAD_STAGED or the driver offers no tensor-map
 * encoder, in which case the CTA's threads copy them (two stages). */
int xpbd_gemm_bf16(const XpbdGemm* g, int32_t n_tile, xpbd_stream_t stream);

/* db[o] = sum_{s < m} dzt[o][s] for o < n_out (BF16 rows of length >= m). */
int xpbd_colsum_bf16(int32_t n_out, int32_t m, const uint16_t* dzt, int32_t ld, float* db, xpbd_stream_t stream);

/* Adam step (Kingma & Ba 2015) on FP32 weights w[rows][cols] with gradient
 * g (row stride ld_g), moments m1, m2, bias correction of step `step`;
 * refreshes the BF16 copy (optional) and the BF16 transposed copy
 * w_bf16_t[cols][ld_t] (optional). */
int xpbd_adam(int32_t rows, int32_t cols, float* w, const float* g, int32_t ld_g, float* m1, float* m2, float lr,
              float beta1, float beta2, float eps, int32_t step, uint16_t* w_bf16, uint16_t* w_bf16_t, int32_t ld_t,
              xpbd_stream_t stream);

/* Mean-squared-error gradient 2 (y - t) / (m n_out) of the valid m x n_out
 * block into the BF16 (m_pad x ld) buffer d (zero elsewhere) and optionally
 * its transpose d_t[ld][ld_dt]; loss[0] += sum (y - t)^2. */
int xpbd_mse_grad(int32_t m, int32_t m_pad, int32_t n_out, int32_t ld, const float* y, int32_t ld_y, const float* t,
                  int32_t ld_t, uint16_t* d, uint16_t* d_t, int32_t ld_dt, float* loss, xpbd_stream_t stream);

/* Static description of the cage for the feature kernel (cage order j). */
typedef struct XpbdCageFeatures {
    int32_t n_cage, m_pad;     /* cage vertices; rows of the feature matrix (>= n_cage) */
    const int32_t* coarse_lib; /* [n_cage] cage order -> coarse library order */
    const int32_t* nbr;        /* [n_cage][6] lattice neighbours (+x,-x,+y,-y,+z,-z of the muscle frame), -1 = none */
    const int32_t* owner;      /* [n_cage] owning muscle */
    const float* act_muscle;   /* [n_muscles] activation of each muscle this frame */
    const int32_t* cage_bone;  /* [n_cage][2] the owner's two end bones */
    const float* cage_w;       /* [n_cage] axial blend weight of the second bone */
    const float* bone_rel;     /* [n_bones][12] frame-to-frame bone motion [R | t], row-major */
    const float* stat;         /* [n_cage][24] static features */
    const float* c_rest4;      /* [n_coarse][4] rest cage (library order) */
    const float* c_target4;    /* [n_coarse][4] restriction of the bone-driven fine targets (library order) */
    const float* norm;         /* [64][2] (mean, 1/std) standardisation of each feature, or NULL */
} XpbdCageFeatures;

/* 64 features per cage vertex into X[m_pad][64] and its transpose Xt[64][m_pad]
 * (BF16): predicted displacement c_pred - c_prev (mm), owner activation,
 * blended bone motion, six neighbours' relative predicted displacement,
 * offsets from the rest cage and to the restricted targets (mm), static rest
 * features. */
int xpbd_cage_features(const XpbdCageFeatures* cf, const float* c_pred4, const float* c_prev4, uint16_t* X,
                       uint16_t* Xt, xpbd_stream_t stream);
/* c_out4[lib j].xyz = c_pred4[lib j].xyz + scale * y[j][0..2]. */
int xpbd_cage_apply(int32_t n_cage, const int32_t* coarse_lib, const float* c_pred4, const float* y, int32_t ldy,
                    float scale, float* c_out4, xpbd_stream_t stream);
/* t[j][0..2] = scale * (c_star4 - c_pred4)[lib j]: the training target. */
int xpbd_cage_target(int32_t n_cage, const int32_t* coarse_lib, const float* c_star4, const float* c_pred4,
                     float scale, float* t, xpbd_stream_t stream);
/* If warm->resid_sq_sum > factor * plain->resid_sq_sum (or the warm state has
 * a non-finite position), pos4 = saved4 and taken[0] += 1. */
int xpbd_fallback_select(int32_t n, const XpbdMetrics* warm, const XpbdMetrics* plain, float factor,
                         const float* saved4, float* pos4, int32_t* taken, xpbd_stream_t stream);

/* Stream capture helpers (a captured substep replays as one graph launch). */
int xpbd_graph_begin(xpbd_stream_t stream);
int xpbd_graph_end(xpbd_stream_t stream, void** exec_out);
int xpbd_graph_launch(void* exec, xpbd_stream_t stream);
int xpbd_graph_destroy(void* exec);

#ifdef __cplusplus
}
#endif
#endif /* XPBD_B200_H */
