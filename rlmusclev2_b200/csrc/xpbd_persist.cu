// Persistent multi-iteration tet pass (xpbd_iterate_persistent).
//
// One cooperative launch runs n_iters Jacobi iterations.  Each CTA keeps its
// tile's vertices (positions, and previous positions for damped materials) in
// shared memory for the whole launch.  Per iteration: project the tile's tets
// into shared accumulators, finish the interior vertices in place, add the
// tile-boundary partial sums to ring slot `cur` of a three-slot global
// accumulator, one grid-wide barrier, then every tile touching a boundary
// vertex finishes it from the complete sum (all of them compute the same
// value from the same inputs).  The owner tile of each boundary vertex clears
// slot `cur + 1`, which was last read two iterations earlier and is next
// filled one iteration later, so one barrier per iteration suffices.  The
// ring phase persists in sync[2] across launches; the slot the next launch
// starts on is the one cleared in this launch's last iteration.
#include <cuda/atomic>
#include <cuda_runtime.h>

#include "xpbd_common.cuh"
#include "xpbd_grid.cuh"
#include "xpbd_tile.cuh"
#include "xpbd_tile_x2.cuh"

using namespace xpbd;

namespace {

constexpr int kThreads = 256;
constexpr size_t kSmemPerVert = 4 * sizeof(float4) + 4 * sizeof(float) + 2 * sizeof(int);  // 88 bytes
// Tiles of at most kFixV vertices put the accumulators and the positions at
// compile-time offsets of the shared block, so the 16 shared atomics and the
// 4 position loads of a tet address their vertex by one register plus an
// immediate (no per-array base register arithmetic).
constexpr int kFixV = 768;

template <bool DAMP, int MINB, int CSET, bool PF, bool X2, bool FIXED = false>
__global__ void __launch_bounds__(kThreads, MINB)
    k_iterate_persistent(const __grid_constant__ XpbdParams prm, const __grid_constant__ XpbdTiles T,
                         const __grid_constant__ XpbdVerts V, const __grid_constant__ XpbdPersist P, int n_iters) {
    extern __shared__ float4 smem[];
    const int tile = P.tile_begin + int(blockIdx.x);
    const int vbeg = T.tile_vptr[tile];
    const int nvt = T.tile_vptr[tile + 1] - vbeg;
    const int nint = T.tile_nint[tile];
    const int own_lo = P.tile_own[tile], own_hi = P.tile_own[tile + 1];
    const int orph_lo = P.tile_end == T.n_tiles ? P.tile_own[T.n_tiles] : V.n;  // last range only
    // Shared layout per tile vertex: position, previous position, attach
    // target, pin target (float4 each), the four accumulator floats, the
    // global id and the vertex flags: 88 bytes.  Everything but the position
    // and the accumulators is constant for the launch.
    const int mtv = T.max_tile_verts;
    float4 *s_pos, *s_prev, *s_att, *s_pin;
    int *s_ax, *s_ay, *s_az, *s_cnt, *s_g, *s_f;
    if constexpr (FIXED) {
        // [4 x kFixV accumulator ints][kFixV positions][prev, attach, pin: mtv each][ids, flags]
        s_ax = reinterpret_cast<int*>(smem);
        s_ay = s_ax + kFixV;
        s_az = s_ay + kFixV;
        s_cnt = s_az + kFixV;
        s_pos = smem + kFixV;
        s_prev = smem + 2 * kFixV;
        s_att = s_prev + mtv;
        s_pin = s_att + mtv;
        s_g = reinterpret_cast<int*>(s_pin + mtv);
        s_f = s_g + mtv;
    } else {
        s_pos = smem;
        s_prev = smem + mtv;
        s_att = smem + 2 * mtv;
        s_pin = smem + 3 * mtv;
        s_ax = reinterpret_cast<int*>(smem + 4 * mtv);
        s_ay = s_ax + mtv;
        s_az = s_ay + mtv;
        s_cnt = s_az + mtv;
        s_g = s_cnt + mtv;
        s_f = s_g + mtv;
    }
    const float inv_scale = 1.f / prm.acc_scale;
    const float4* pos4 = reinterpret_cast<const float4*>(V.pos);
    const float4* prev4 = reinterpret_cast<const float4*>(V.pprev);
    float4* pos4w = reinterpret_cast<float4*>(V.pos);
    float4* ring = reinterpret_cast<float4*>(P.ring);
    const size_t nv = size_t(V.n);
    const uint32_t phase0 = P.sync[2];
    const bool nsync = P.nbr_ptr != nullptr;
    GridBarrier bar = {nullptr, 0u, 0u};
    uint32_t c0 = 0;
    const int32_t* nbr = nullptr;
    int n_nbr = 0;
    if (nsync) {
        c0 = __ldcg(P.tile_cnt + tile);
        nbr = P.nbr_idx + P.nbr_ptr[tile];
        n_nbr = P.nbr_ptr[tile + 1] - P.nbr_ptr[tile];
    } else {
        bar = grid_barrier_begin(P.sync);
    }
    const uint32_t ops = XPBD_APPLY_ATTACH | XPBD_APPLY_DIVIDE | XPBD_APPLY_PIN;
    __shared__ float s_arap_at[XPBD_MAX_MATERIALS];
    __shared__ int s_defer[2 + kDeferCap];
    if (threadIdx.x == 0) s_defer[0] = s_defer[1] = 0;
    fill_arap_at(prm, s_arap_at);
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int i = threadIdx.x; i < nvt; i += blockDim.x) {
        const int g = T.tile_verts[vbeg + i];
        const int f = V.vflags ? V.vflags[g] : 0;
        s_g[i] = g;
        s_f[i] = f;
        s_pos[i] = pos4[g];
        s_prev[i] = prev4 ? prev4[g] : z4;
        s_att[i] = (f & XPBD_VF_ATTACH_MASK) ? reinterpret_cast<const float4*>(V.attach_target)[g] : z4;
        s_pin[i] = (f & XPBD_VF_PIN) ? reinterpret_cast<const float4*>(V.pin_target)[g] : z4;
    }
    // The accumulators start zeroed and each vertex's are zeroed again where
    // they are read (the finish or the boundary push), so no clearing pass
    // runs between iterations.
    for (int i = threadIdx.x; i < nvt; i += blockDim.x) {
        s_ax[i] = 0;
        s_ay[i] = 0;
        s_az[i] = 0;
        s_cnt[i] = 0;
    }
    // Finish of tile vertex i from its sum a; only the staged data its flags use is read.
    auto finish_local = [&](int i, float4 a) {
        const int f = s_f[i];
        float4 at = z4, pv = z4, pin = z4;
        if (f & XPBD_VF_ATTACH_MASK) {
            at = s_att[i];
            pv = s_prev[i];
        }
        if (f & XPBD_VF_PIN) pin = s_pin[i];
        float4 pp = s_pos[i];
        finish_core(prm, f, at, pv, pin, pp, a, ops);
        s_pos[i] = pp;
    };
    auto take_acc = [&](int i) {
        const float4 a = tile_acc(s_ax, s_ay, s_az, s_cnt, i, inv_scale);
        s_ax[i] = 0;
        s_ay[i] = 0;
        s_az[i] = 0;
        s_cnt[i] = 0;
        return a;
    };
    for (int it = 0; it < n_iters; ++it) {
        const uint32_t cur = (phase0 + uint32_t(it)) % 3u, nxt = (phase0 + uint32_t(it) + 1u) % 3u;
        float4* rc = ring + cur * nv;
        float4* rn = ring + nxt * nv;
        __syncthreads();  // staged or finished positions, zeroed accumulators
        if constexpr (X2 && CSET != CSET_FULL && !DAMP)
            project_tile_tets_x2<CSET == CSET_VOL>(prm, T, tile, s_pos, s_ax, s_ay, s_az, s_cnt, s_arap_at);
        else
            project_tile_tets<DAMP, CSET, PF>(prm, T, tile, s_pos, s_prev, s_ax, s_ay, s_az, s_cnt, s_arap_at,
                                              s_defer, it & 1);
        __syncthreads();
        // boundary partial sums first, so their L2 atomics overlap the interior finish
        for (int i = nint + threadIdx.x; i < nvt; i += blockDim.x) {
            const int g = s_g[i];
            const float4 a = take_acc(i);
            if (a.w != 0.f) atomicAdd(&rc[g], a);
            if (g >= own_lo && g < own_hi) rn[g] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        for (int i = threadIdx.x; i < nint; i += blockDim.x) finish_local(i, take_acc(i));
        // vertices in no tet: attach and pin only, each handled by one thread
        for (int g = orph_lo + int(blockIdx.x) * blockDim.x + threadIdx.x; g < V.n; g += gridDim.x * blockDim.x) {
            float4 pp = pos4[g];
            finish_vertex(prm, V, g, pp, make_float4(0.f, 0.f, 0.f, 0.f), ops);
            pos4w[g] = pp;
        }
        if (nsync)
            neighbour_sync(P.tile_cnt, nbr, n_nbr, tile, c0 + uint32_t(it) + 1u, P.status);
        else
            grid_barrier(bar, P.status);
        for (int i = nint + threadIdx.x; i < nvt; i += blockDim.x) finish_local(i, __ldcg(&rc[s_g[i]]));
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nvt; i += blockDim.x) {
        const int g = s_g[i];
        if (i < nint || (g >= own_lo && g < own_hi)) pos4w[g] = s_pos[i];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) P.sync[2] = (phase0 + uint32_t(n_iters)) % 3u;
    if (!nsync) grid_barrier_end(P.sync, bar);
}

uint32_t material_union(const XpbdParams* p) {
    uint32_t u = 0;
    for (int i = 0; i < p->n_materials; ++i) u |= p->materials[i].flags;
    return u;
}

template <bool DAMP, int MINB, int CSET, bool PF, bool X2 = false, bool FIXED = false>
int launch_v(const XpbdParams* prm, const XpbdTiles* T, const XpbdVerts* V, const XpbdPersist* P, int n_iters,
             cudaStream_t s, bool query_only, int* fits) {
    auto kern = k_iterate_persistent<DAMP, MINB, CSET, PF, X2, FIXED>;
    const size_t smem = FIXED ? size_t(kFixV) * (4 * sizeof(int) + sizeof(float4)) +
                                    size_t(T->max_tile_verts) * (3 * sizeof(float4) + 2 * sizeof(int))
                              : size_t(T->max_tile_verts) * kSmemPerVert;
    if (smem > kSmemOptIn &&
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess)
        return cuda_check("xpbd_iterate_persistent: smem attribute");
    int dev = 0, n_sm = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, smem) != cudaSuccess)
        return cuda_check("xpbd_iterate_persistent: occupancy");
    const int64_t slots = int64_t(per_sm) * n_sm;
    if (query_only) {
        fits[0] = slots >= T->n_tiles ? 1 : 0;
        fits[1] = int(slots);
        return XPBD_OK;
    }
    const int ntl = P->tile_end - P->tile_begin;
    if (ntl > slots) return fail(XPBD_ERR_LIMIT, "xpbd_iterate_persistent: tiles exceed the resident CTA slots");
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(ntl);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (cudaLaunchKernelEx(&cfg, kern, *prm, *T, *V, *P, n_iters) != cudaSuccess)
        return cuda_check("xpbd_iterate_persistent: launch");
    return cuda_check("xpbd_iterate_persistent");
}

// Same instance choice as the per-iteration pass.
int dispatch(const XpbdParams* prm, const XpbdTiles* T, const XpbdVerts* V, const XpbdPersist* P, int n_iters,
             cudaStream_t s, bool query_only, int* fits) {
    const uint32_t u = material_union(prm);
    bool damp = false;
    for (int i = 0; i < prm->n_materials; ++i)
        if (prm->materials[i].flags & XPBD_MAT_DAMPED) damp = true;
    const bool flip = (prm->tile_variant & 1) != 0;
    const bool pf = (prm->tile_variant & 4) != 0;
    // tile_variant bit 4: the runtime shared layout even for small tiles
    const bool fixed = T->max_tile_verts <= kFixV && !(prm->tile_variant & 16);
#define XPBD_LAUNCH(D, M, C) \
    (pf ? launch_v<D, M, C, true>(prm, T, V, P, n_iters, s, query_only, fits) \
        : (fixed ? launch_v<D, M, C, false, false, true>(prm, T, V, P, n_iters, s, query_only, fits) \
                 : launch_v<D, M, C, false>(prm, T, V, P, n_iters, s, query_only, fits)))
    if (u & XPBD_MAT_SNH) {
        if (damp) return flip ? XPBD_LAUNCH(true, 3, CSET_FULL) : XPBD_LAUNCH(true, 2, CSET_FULL);
        return flip ? XPBD_LAUNCH(false, 3, CSET_FULL) : XPBD_LAUNCH(false, 2, CSET_FULL);
    }
    if (u & XPBD_MAT_VOLUME) {
        if (damp) return flip ? XPBD_LAUNCH(true, 3, CSET_VOL) : XPBD_LAUNCH(true, 2, CSET_VOL);
        if (prm->tile_variant & 8) return launch_v<false, 2, CSET_VOL, false, true>(prm, T, V, P, n_iters, s, query_only, fits);
        return flip ? XPBD_LAUNCH(false, 3, CSET_VOL) : XPBD_LAUNCH(false, 2, CSET_VOL);
    }
    // tile_variant bit 3: the two-tet packed pass (2 CTAs/SM at up to 128
    // registers; slower on B200, measured)
    if (prm->tile_variant & 8) return launch_v<false, 2, CSET_LIGHT, false, true>(prm, T, V, P, n_iters, s, query_only, fits);
    return flip ? XPBD_LAUNCH(false, 2, CSET_LIGHT) : XPBD_LAUNCH(false, 3, CSET_LIGHT);
#undef XPBD_LAUNCH
}

}  // namespace

extern "C" int xpbd_iterate_persistent(const XpbdParams* prm, const XpbdTiles* tiles, const XpbdVerts* v,
                                       const XpbdPersist* ps, int32_t n_iters, xpbd_stream_t stream) {
    if (!prm || !tiles || !v || !ps) return fail(XPBD_ERR_ARG, "xpbd_iterate_persistent: null argument");
    if (n_iters < 0) return fail(XPBD_ERR_ARG, "xpbd_iterate_persistent: n_iters < 0");
    if (n_iters == 0) return XPBD_OK;
    // barrier counters reach n_iters x grid size within one launch
    if (n_iters > (1 << 20)) return fail(XPBD_ERR_LIMIT, "xpbd_iterate_persistent: n_iters > 2^20");
    if (!v->pos || v->n <= 0 || !tiles->tile_vptr || !tiles->tile_nint || !tiles->tile_tptr || !tiles->tile_verts ||
        !tiles->tet_q || !tiles->tet_b0 || !tiles->tet_b1 || !tiles->tet_b2 || tiles->n_tiles <= 0)
        return fail(XPBD_ERR_ARG, "xpbd_iterate_persistent: tiles/verts");
    if (!ps->tile_own || !ps->ring || !ps->sync || !ps->status)
        return fail(XPBD_ERR_ARG, "xpbd_iterate_persistent: XpbdPersist pointers");
    if ((ps->nbr_ptr == nullptr) != (ps->nbr_idx == nullptr) || (ps->nbr_ptr == nullptr) != (ps->tile_cnt == nullptr))
        return fail(XPBD_ERR_ARG, "xpbd_iterate_persistent: nbr_ptr, nbr_idx and tile_cnt must be set together");
    XpbdPersist P = *ps;
    if (P.tile_begin == 0 && P.tile_end == 0) P.tile_end = tiles->n_tiles;
    if (P.tile_begin < 0 || P.tile_end > tiles->n_tiles || P.tile_begin >= P.tile_end)
        return fail(XPBD_ERR_ARG, "xpbd_iterate_persistent: tile range");
    if (!aligned16(v->pos) || !aligned16(ps->ring)) return fail(XPBD_ERR_ALIGN, "xpbd_iterate_persistent: alignment");
    if (tiles->max_tile_verts > XPBD_MAX_TILE_VERTS) return fail(XPBD_ERR_LIMIT, "xpbd_iterate_persistent: tile size");
    if (prm->n_materials < 1 || prm->n_materials > XPBD_MAX_MATERIALS)
        return fail(XPBD_ERR_ARG, "xpbd_iterate_persistent: n_materials");
    if (!(prm->acc_scale > 0.f) || !(prm->acc_scale < 3.0e38f))
        return fail(XPBD_ERR_ARG, "xpbd_iterate_persistent: acc_scale must be a finite value > 0");
    bool aniso = false, damp = false;
    for (int i = 0; i < prm->n_materials; ++i) {
        aniso |= (prm->materials[i].flags & XPBD_MAT_ANISO) != 0;
        damp |= (prm->materials[i].flags & XPBD_MAT_DAMPED) != 0;
    }
    if (aniso && (!tiles->tet_fiber || !tiles->tet_act))
        return fail(XPBD_ERR_ARG, "xpbd_iterate_persistent: aniso materials need tet_fiber and tet_act");
    if (damp && !v->pprev) return fail(XPBD_ERR_ARG, "xpbd_iterate_persistent: damped materials need pprev");
    return dispatch(prm, tiles, v, &P, n_iters, (cudaStream_t)stream, false, nullptr);
}

extern "C" int xpbd_persistent_fits(const XpbdParams* prm, const XpbdTiles* tiles, int32_t* fits, int32_t* slots) {
    if (!prm || !tiles || !fits) return fail(XPBD_ERR_ARG, "xpbd_persistent_fits: null argument");
    if (prm->n_materials < 1 || prm->n_materials > XPBD_MAX_MATERIALS)
        return fail(XPBD_ERR_ARG, "xpbd_persistent_fits: n_materials");
    int f[2] = {0, 0};
    const int rc = dispatch(prm, tiles, nullptr, nullptr, 0, nullptr, true, f);
    *fits = f[0];
    if (slots) *slots = f[1];
    return rc;
}
