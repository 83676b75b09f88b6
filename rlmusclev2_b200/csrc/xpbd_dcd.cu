// Triangle-triangle discrete collision detection (DCD) for sm_100a.
//
// Broadphase: per-triangle AABBs padded by the thickness, 30-bit Morton codes
// of their centres, a stable LSD radix sort (8-bit digits, per-warp ranking
// with __match_any_sync), a linear BVH built with Karras' method ("Maximizing
// Parallelism in the Construction of BVHs, Octrees, and k-d Trees", HPG 2012)
// and refitted bottom-up with per-node arrival counters; then a two-pass
// traversal (count, exclusive scan, fill) that lists the AABB-overlapping
// pairs (i, j > i) of every triangle in a deterministic order.
//
// Narrowphase / response / apply restate the reference's UDCF kernels
// (collision/udcf/kernel.py:164-474, 713-822): Moller interval rejection,
// VF/FV/EE candidate depths C1/C2, smaller-positive wins (tie -> C2), equal
// push of the three vertices of each movable face, friction on the
// bary-weighted tangential displacement, Jacobi averaging.
#include <cuda_runtime.h>

#include <algorithm>

#include "xpbd_common.cuh"
#include "xpbd_device.cuh"
#include "xpbd_grid.cuh"

using namespace xpbd;

namespace {

constexpr int kSortThreads = 1024;  // keys per scatter round; the sort's CTA size
constexpr int kScanItems = 4;     // consecutive elements per thread in the block scan
constexpr int kScanBlock = 1024 * kScanItems;
constexpr int kStack = 64;
constexpr int kSlots = 16;  // partners a query keeps from the counting pass
constexpr float kThresh = 1.0e-5f;  // udcf/kernel.py:40 THRESH

struct Aabb {
    float3 lo, hi;
};

__device__ __forceinline__ float4 ld4(const float* p, int i) { return reinterpret_cast<const float4*>(p)[i]; }

// ws_nodes layout (float4 units): internal node records [4 (n-1)), then the
// leaf boxes in Morton order [2 n), then the leaf boxes in triangle order
// [2 n).  Record i holds its two children: lo_a (w: last Morton position
// under a), hi_a (w: a's node id), lo_b, hi_b; node ids >= n-1 are leaves
// (position id - (n-1)).  A visit is one 64-byte load.
__host__ __device__ __forceinline__ int64_t sorted_leaf_base(int n) { return int64_t(4) * (n - 1); }
__host__ __device__ __forceinline__ int64_t tri_leaf_base(int n) { return int64_t(4) * (n - 1) + 2 * int64_t(n); }

__device__ __forceinline__ uint32_t spread10(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

// ---------------------------------------------------------------- AABBs
// KEYS = false (refit-only broadphase): boxes only; the Morton keys and the
// sorted order of the last rebuild are kept.
template <bool KEYS>
__global__ void k_tri_aabb(XpbdDcd D, const float* __restrict__ pos4) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.n_tris) return;
    const int a = D.tris[3 * i], b = D.tris[3 * i + 1], c = D.tris[3 * i + 2];
    const float3 pa = f3(ld4(pos4, a)), pb = f3(ld4(pos4, b)), pc = f3(ld4(pos4, c));
    const float t = D.thickness;
    // tri_aabb_kernel (udcf/kernel.py:917-934)
    const float3 lo = make_float3(fminf(fminf(pa.x, pb.x), pc.x) - t, fminf(fminf(pa.y, pb.y), pc.y) - t,
                                  fminf(fminf(pa.z, pb.z), pc.z) - t);
    const float3 hi = make_float3(fmaxf(fmaxf(pa.x, pb.x), pc.x) + t, fmaxf(fmaxf(pa.y, pb.y), pc.y) + t,
                                  fmaxf(fmaxf(pa.z, pb.z), pc.z) + t);
    float4* tri_box = reinterpret_cast<float4*>(D.ws_nodes) + tri_leaf_base(D.n_tris);
    tri_box[2 * i] = make_float4(lo.x, lo.y, lo.z, 0.f);
    tri_box[2 * i + 1] = make_float4(hi.x, hi.y, hi.z, 0.f);
    if (!KEYS) return;
    const float3 cen = make_float3(0.5f * (lo.x + hi.x), 0.5f * (lo.y + hi.y), 0.5f * (lo.z + hi.z));
    float q[3] = {cen.x, cen.y, cen.z};
    uint32_t code = 0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float ext = fmaxf(D.box_hi[k] - D.box_lo[k], 1e-30f);
        float u = (q[k] - D.box_lo[k]) / ext * 1023.f;
        u = fminf(fmaxf(u, 0.f), 1023.f);
        code |= spread10(uint32_t(u)) << k;
    }
    D.ws_keys[i] = code;
    D.ws_vals[i] = i;
}

// ---------------------------------------------------------- radix sort
// Exclusive scan in three launches: per-block scans of kScanBlock elements
// (each thread a run of kScanItems, warp shuffles across threads) leaving
// block totals in sums[], one CTA scanning sums[], and a launch adding each
// block's offset.  total (optional) receives the sum of all elements.
__device__ __forceinline__ int block_excl_scan(int v, int* warp_sums, int* block_total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[w] = x;
    __syncthreads();
    if (w == 0) {
        int t = lane < int(blockDim.x >> 5) ? warp_sums[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        warp_sums[lane] = t;
    }
    __syncthreads();
    const int incl = x + (w > 0 ? warp_sums[w - 1] : 0);
    if (block_total && threadIdx.x == blockDim.x - 1) *block_total = incl;
    return incl - v;
}

__global__ void __launch_bounds__(1024) k_scan_blocks(int* __restrict__ a, int n, int* __restrict__ sums) {
    __shared__ int warp_sums[32];
    __shared__ int total;
    const int base = blockIdx.x * kScanBlock + threadIdx.x * kScanItems;
    int v[kScanItems];
    int run = 0;
#pragma unroll
    for (int q = 0; q < kScanItems; ++q) {
        v[q] = base + q < n ? a[base + q] : 0;
        run += v[q];
    }
    int off = block_excl_scan(run, warp_sums, &total);
#pragma unroll
    for (int q = 0; q < kScanItems; ++q) {
        if (base + q < n) a[base + q] = off;
        off += v[q];
    }
    __syncthreads();
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(1024) k_scan_sums(int* __restrict__ sums, int nb, int* __restrict__ total) {
    __shared__ int warp_sums[32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int b0 = 0; b0 < nb; b0 += blockDim.x) {
        const int i = b0 + threadIdx.x;
        const int v = i < nb ? sums[i] : 0;
        __shared__ int round_total;
        const int e = block_excl_scan(v, warp_sums, &round_total) + carry;
        if (i < nb) sums[i] = e;
        __syncthreads();
        if (threadIdx.x == 0) carry += round_total;
        __syncthreads();
    }
    if (total && threadIdx.x == 0) *total = carry;
}

__global__ void __launch_bounds__(1024) k_scan_add(int* __restrict__ a, int n, const int* __restrict__ sums) {
    const int add = sums[blockIdx.x];
    const int base = blockIdx.x * kScanBlock + threadIdx.x * kScanItems;
#pragma unroll
    for (int q = 0; q < kScanItems; ++q)
        if (base + q < n) a[base + q] += add;
}

void scan_excl(int* a, int n, int* total, int* scratch, cudaStream_t s) {
    const int nb = (n + kScanBlock - 1) / kScanBlock;
    k_scan_blocks<<<nb, 1024, 0, s>>>(a, n, scratch);
    k_scan_sums<<<1, 1024, 0, s>>>(scratch, nb, total);
    if (nb > 1) k_scan_add<<<nb, 1024, 0, s>>>(a, n, scratch);
}

// Radix sort of (Morton key, triangle id), 4 passes of 8 bits, in one
// cooperative launch: CTA b owns the contiguous chunk [b C, (b+1) C) of the
// pass input.  Per pass: (A) chunk histogram -> hist[b][256]; grid barrier;
// (B) every CTA sums the histograms itself (digit totals, and the counts of
// the chunks before its own) and scans the totals over digits, giving its
// first output slot per digit; (C) stable scatter in rounds of kSortThreads
// keys: warps rank equal digits with __match_any_sync, per-digit prefix over
// the warps in shared memory; grid barrier before the next pass reads.
// Even pass count: the sorted data ends in ws_keys/ws_vals.
__device__ __forceinline__ int add_excl_over_warps(int (*wcnt)[256], int d, int run) {
    for (int ww = 0; ww < kSortThreads / 32; ++ww) {
        const int c = wcnt[ww][d];
        wcnt[ww][d] = run;
        run += c;
    }
    return run;
}

__global__ void __launch_bounds__(kSortThreads) k_sort_coop(XpbdDcd D, int chunk, uint32_t* sync) {
    __shared__ int wcnt[kSortThreads / 32][256];
    __shared__ int run[256];
    __shared__ int part[kSortThreads / 256][256];
    __shared__ int warp_sums[32];
    const int n = D.n_tris, G = gridDim.x, b = blockIdx.x;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int beg = min(n, b * chunk), end = min(n, beg + chunk);
    int* hist = D.ws_hist;  // [G][256]
    uint32_t* ks = D.ws_keys;
    int32_t* vs = D.ws_vals;
    uint32_t* kd = D.ws_keys2;
    int32_t* vd = D.ws_vals2;
    GridBarrier bar = grid_barrier_begin(sync);
    for (int pass = 0; pass < 4; ++pass) {
        const int shift = 8 * pass;
        // (A) chunk histogram
        if (threadIdx.x < 256) run[threadIdx.x] = 0;
        __syncthreads();
        for (int i = beg + int(threadIdx.x); i < end; i += kSortThreads) {
            const int dig = int((ks[i] >> shift) & 255u);
            const unsigned peers = __match_any_sync(__activemask(), dig);
            if ((peers & ((1u << lane) - 1u)) == 0) atomicAdd(&run[dig], __popc(peers));
        }
        __syncthreads();
        if (threadIdx.x < 256) hist[b * 256 + threadIdx.x] = run[threadIdx.x];
        grid_barrier(bar, D.status);
        // (B) first output slot of each digit for this chunk
        {
            const int d = threadIdx.x & 255, q = threadIdx.x >> 8;
            constexpr int kQ = kSortThreads / 256;
            int tot = 0, pre = 0;
            // the CTAs' counts are independent L2 reads: unrolled so that several
            // are in flight at once instead of one latency per CTA
#pragma unroll 8
            for (int bb = q; bb < G; bb += kQ) {
                const int h = __ldcg(&hist[bb * 256 + d]);
                tot += h;
                pre += bb < b ? h : 0;
            }
            part[q][d] = tot;
            wcnt[q][d] = pre;
            __syncthreads();
            int t_all = 0, p_all = 0;
            if (q == 0) {
                for (int k = 0; k < kQ; ++k) {
                    t_all += part[k][d];
                    p_all += wcnt[k][d];
                }
            }
            const int base = block_excl_scan(q == 0 ? t_all : 0, warp_sums, nullptr);
            if (q == 0) run[d] = base + p_all;
            __syncthreads();
        }
        // (C) stable scatter
        for (int r = beg; r < end; r += kSortThreads) {
            for (int k = threadIdx.x; k < (kSortThreads / 32) * 256; k += kSortThreads) (&wcnt[0][0])[k] = 0;
            __syncthreads();
            const int i = r + int(threadIdx.x);
            const bool valid = i < end;
            const uint32_t key = valid ? ks[i] : 0u;
            const int dig = valid ? int((key >> shift) & 255u) : 256;
            const unsigned peers = __match_any_sync(0xffffffffu, dig);
            const int lrank = __popc(peers & ((1u << lane) - 1u));
            if (valid && lrank == 0) wcnt[w][dig] = __popc(peers);
            __syncthreads();
            if (threadIdx.x < 256) run[threadIdx.x] = add_excl_over_warps(wcnt, threadIdx.x, run[threadIdx.x]);
            __syncthreads();
            const int dst = valid ? wcnt[w][dig] + lrank : -1;
            if (dst >= 0 && dst < n) {  // always, unless a barrier gave up (status bit set)
                kd[dst] = key;
                vd[dst] = vs[i];
            }
            __syncthreads();
        }
        if (pass < 3) grid_barrier(bar, D.status);
        uint32_t* tk = ks; ks = kd; kd = tk;
        int32_t* tv = vs; vs = vd; vd = tv;
    }
    grid_barrier_end(sync, bar);
}

// ---------------------------------------------------------- Karras build
__device__ __forceinline__ int delta(const uint32_t* k, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    const uint32_t a = k[i], b = k[j];
    if (a == b) return 32 + __clz(uint32_t(i) ^ uint32_t(j));
    return __clz(a ^ b);
}

// Box of the sorted leaves [a, b): leaf boxes at the ends, 32-leaf block boxes
// (ws_bbox[0, nb32)) and 1024-leaf block boxes (ws_bbox[nb32, ...)) between.
// Independent loads, no dependence on other internal nodes: the whole
// hierarchy's boxes come out of the build launch without a bottom-up refit.
struct Box {
    float4 lo, hi;
    __device__ __forceinline__ void add(const float4* p, int k) {
        const float4 l = p[2 * k], h = p[2 * k + 1];
        lo.x = fminf(lo.x, l.x), lo.y = fminf(lo.y, l.y), lo.z = fminf(lo.z, l.z);
        hi.x = fmaxf(hi.x, h.x), hi.y = fmaxf(hi.y, h.y), hi.z = fmaxf(hi.z, h.z);
    }
};

__device__ __forceinline__ void add_run(Box& bx, const float4* p, int a, int b) {
#pragma unroll 4
    for (int k = a; k < b; ++k) bx.add(p, k);
}

__device__ Box range_box(const XpbdDcd& D, int a, int b) {
    const int n = D.n_tris;
    const float4* leaves = reinterpret_cast<const float4*>(D.ws_nodes) + sorted_leaf_base(n);
    const float4* b32 = reinterpret_cast<const float4*>(D.ws_bbox);
    const float4* b1k = b32 + 2 * ((n + 31) / 32);
    Box bx;
    bx.lo = make_float4(INFINITY, INFINITY, INFINITY, 0.f);
    bx.hi = make_float4(-INFINITY, -INFINITY, -INFINITY, 0.f);
    if (b - a <= 64) {
        add_run(bx, leaves, a, b);
        return bx;
    }
    const int a1 = (a + 31) >> 5, e1 = b >> 5;  // whole 32-leaf blocks [a1, e1)
    add_run(bx, leaves, a, a1 << 5);
    add_run(bx, leaves, e1 << 5, b);
    if (e1 - a1 <= 64) {
        add_run(bx, b32, a1, e1);
        return bx;
    }
    const int a2 = (a1 + 31) >> 5, e2 = e1 >> 5;  // whole 1024-leaf blocks [a2, e2)
    add_run(bx, b32, a1, a2 << 5);
    add_run(bx, b32, e2 << 5, e1);
    add_run(bx, b1k, a2, e2);
    return bx;
}

// Half `side` of internal node i's record: the box of the child covering
// [lo, g] (side 0) or [g + 1, hi] (side 1), its last Morton position, its id.
__device__ __forceinline__ void write_child(const XpbdDcd& D, int i, int side, int lo, int g, int hi) {
    const int n = D.n_tris;
    const int first = side ? g + 1 : lo, last = side ? hi : g;
    const int id = (first == last) ? (n - 1 + first) : (side ? g + 1 : g);
    const Box bx = range_box(D, first, last + 1);
    float4* rec = reinterpret_cast<float4*>(D.ws_nodes) + 4 * int64_t(i) + 2 * side;
    rec[0] = make_float4(bx.lo.x, bx.lo.y, bx.lo.z, __int_as_float(last));
    rec[1] = make_float4(bx.hi.x, bx.hi.y, bx.hi.z, __int_as_float(id));
}

// Karras (2012) hierarchy over the sorted keys.  Two threads per internal
// node i (adjacent lanes) both run its split search; thread `side` then
// writes child `side`'s half of record i: box from the child's leaf range,
// last Morton position, node id.  Two threads halve the range-box work per
// thread and double the warps in flight: the launch is latency-bound.
__global__ void k_build(XpbdDcd D) {
    const int n = D.n_tris;
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = gid >> 1, side = gid & 1;
    if (i >= n - 1) return;
    const uint32_t* k = D.ws_keys;
    const int d = (delta(k, n, i, i + 1) - delta(k, n, i, i - 1)) >= 0 ? 1 : -1;
    const int dmin = delta(k, n, i, i - d);
    int lmax = 2;
    while (lmax < 2 * n && delta(k, n, i, i + lmax * d) > dmin) lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
        if (delta(k, n, i, i + (l + t) * d) > dmin) l += t;
    const int j = i + l * d;
    const int dnode = delta(k, n, i, j);
    int s = 0;
    int t = l;
    do {
        t = (t + 1) >> 1;
        if (delta(k, n, i, i + (s + t) * d) > dnode) s += t;
    } while (t > 1);
    const int g = i + s * d + min(d, 0);
    const int lo = min(i, j), hi = max(i, j);
    if (side == 0) reinterpret_cast<int4*>(D.ws_split)[i] = make_int4(lo, g, hi, 0);
    write_child(D, i, side, lo, g, hi);
}

// Refit-only broadphase: the hierarchy of the last rebuild (leaf range and
// split per internal node in ws_split) over the leaves in that rebuild's
// Morton order, boxes recomputed from the current leaf boxes.  The pair set
// does not depend on the hierarchy, only the traversal cost does.
__global__ void k_refit_ranges(XpbdDcd D) {
    const int n = D.n_tris;
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = gid >> 1, side = gid & 1;
    if (i >= n - 1) return;
    const int4 r = reinterpret_cast<const int4*>(D.ws_split)[i];
    write_child(D, i, side, r.x, r.y, r.z);
}

// Leaves were written in triangle order; the build wants them in Morton order.  A CTA of 1024 threads covers 1024
// consecutive leaves and also writes their 32- and 1024-leaf block boxes.
__device__ __forceinline__ void warp_box(float4& lo, float4& hi) {
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
        lo.x = fminf(lo.x, __shfl_xor_sync(0xffffffffu, lo.x, o));
        lo.y = fminf(lo.y, __shfl_xor_sync(0xffffffffu, lo.y, o));
        lo.z = fminf(lo.z, __shfl_xor_sync(0xffffffffu, lo.z, o));
        hi.x = fmaxf(hi.x, __shfl_xor_sync(0xffffffffu, hi.x, o));
        hi.y = fmaxf(hi.y, __shfl_xor_sync(0xffffffffu, hi.y, o));
        hi.z = fmaxf(hi.z, __shfl_xor_sync(0xffffffffu, hi.z, o));
    }
}

__global__ void __launch_bounds__(1024) k_permute_leaves(XpbdDcd D) {
    __shared__ float4 s_box[32][2];
    const int n = D.n_tris;
    const int s = blockIdx.x * 1024 + threadIdx.x;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    float4 lo = make_float4(INFINITY, INFINITY, INFINITY, 0.f), hi = make_float4(-INFINITY, -INFINITY, -INFINITY, 0.f);
    if (s < n) {
        const int tri = D.ws_vals[s];
        const float4* src = reinterpret_cast<const float4*>(D.ws_nodes) + tri_leaf_base(n);
        float4* dst = reinterpret_cast<float4*>(D.ws_nodes) + sorted_leaf_base(n);
        lo = src[2 * tri];
        hi = src[2 * tri + 1];
        dst[2 * s] = lo;
        dst[2 * s + 1] = hi;
    }
    warp_box(lo, hi);
    float4* b32 = reinterpret_cast<float4*>(D.ws_bbox);
    if (lane == 0 && s < n) {
        b32[2 * (s >> 5)] = lo;
        b32[2 * (s >> 5) + 1] = hi;
    }
    if (lane == 0) {
        s_box[w][0] = lo;
        s_box[w][1] = hi;
    }
    __syncthreads();
    if (w == 0) {
        lo = s_box[lane][0];
        hi = s_box[lane][1];
        warp_box(lo, hi);
        if (lane == 0) {
            float4* b1k = b32 + 2 * ((n + 31) / 32);
            b1k[2 * blockIdx.x] = lo;
            b1k[2 * blockIdx.x + 1] = hi;
        }
    }
}

// ------------------------------------------------------------ traversal
__device__ __forceinline__ bool overlap(float4 alo, float4 ahi, float4 blo, float4 bhi) {
    return !(alo.x > bhi.x || blo.x > ahi.x || alo.y > bhi.y || blo.y > ahi.y || alo.z > bhi.z || blo.z > ahi.z);
}

// broadphase_find_pairs_bvh_kernel rules (udcf/kernel.py:937-981): j > i,
// static-static never, movable-self only when allowed and sharing no vertex.
__device__ __forceinline__ bool pair_ok(const XpbdDcd& D, int i, int j) {
    if (j <= i) return false;
    const int gi = D.tri_group ? D.tri_group[i] : 0, gj = D.tri_group ? D.tri_group[j] : 0;
    if (gi == 1 && gj == 1) return false;
    if (gi == 0 && gj == 0) {
        if (!D.allow_self) return false;
        const int a0 = D.tris[3 * i], a1 = D.tris[3 * i + 1], a2 = D.tris[3 * i + 2];
        const int b0 = D.tris[3 * j], b1 = D.tris[3 * j + 1], b2 = D.tris[3 * j + 2];
        if (a0 == b0 || a0 == b1 || a0 == b2 || a1 == b0 || a1 == b1 || a1 == b2 || a2 == b0 || a2 == b1 || a2 == b2)
            return false;
    }
    return true;
}

// Thread t queries the triangle at Morton position t against the leaves at
// later positions only: every unordered overlapping pair is met once, by the
// query that comes first in Morton order, and subtrees whose last position
// (kept in the node's lo.w) is <= t are skipped whole.  A warp's queries are
// spatially close and walk similar paths.  Both children are tested before
// descending; one stack entry per level with two live children.
// The counting pass keeps the first kSlots partners in ws_slots; the fill
// pass copies those and re-traverses only queries with more partners.
// Pairs are written as (min, max) triangle id, grouped by query position.
__device__ __forceinline__ bool live(const float4& qlo, const float4& qhi, const float4& lo, const float4& hi, int t) {
    return __float_as_int(lo.w) > t && overlap(qlo, qhi, lo, hi);
}

template <bool FILL>
__device__ __forceinline__ void emit_leaf(const XpbdDcd& D, int i, int leaf_pos, int t, int& cnt, int& out) {
    const int j = D.ws_vals[leaf_pos];
    const int a = min(i, j), b = max(i, j);
    if (!pair_ok(D, a, b)) return;
    if (FILL) {
        if (out < D.max_pairs) reinterpret_cast<int2*>(D.pairs)[out] = make_int2(a, b);
        ++out;
    } else {
        if (cnt < kSlots) D.ws_slots[int64_t(cnt) * D.n_tris + t] = j;
        ++cnt;
    }
}

template <bool FILL>
__global__ void __launch_bounds__(128) k_traverse(XpbdDcd D) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = D.n_tris;
    if (t >= n) return;
    if (*D.status & XPBD_STATUS_BARRIER_TIMEOUT) return;  // the sort gave up: no valid tree
    const int i = D.ws_vals[t];
    int cnt = 0, out = 0;
    if (FILL) {
        out = D.ws_count[t];
        const int end = t + 1 < n ? D.ws_count[t + 1] : *D.ws_total;
        const int c = end - out;
        if (c <= kSlots) {
            for (int k = 0; k < c; ++k, ++out) {
                if (out >= D.max_pairs) break;
                const int j = D.ws_slots[int64_t(k) * n + t];
                reinterpret_cast<int2*>(D.pairs)[out] = make_int2(min(i, j), max(i, j));
            }
            return;
        }
    }
    if (n > 1) {
        const float4* recs = reinterpret_cast<const float4*>(D.ws_nodes);
        const float4* tri_box = recs + tri_leaf_base(n);
        const float4 qlo = tri_box[2 * i], qhi = tri_box[2 * i + 1];
        int stack[kStack];
        int sp = 0;
        int node = 0;  // the root (its own box is never needed: its record tests both children)
        for (int visits = 0;; ++visits) {
            if (visits >= n) {  // more internal nodes than the tree has: not a tree
                atomicOr(D.status, XPBD_STATUS_STACK_OVERFLOW);
                break;
            }
            const float4* r = recs + 4 * int64_t(node);
            const float4 alo = r[0], ahi = r[1], blo = r[2], bhi = r[3];
            const int ca = __float_as_int(ahi.w), cb = __float_as_int(bhi.w);
            const bool la = live(qlo, qhi, alo, ahi, t);
            const bool lb = live(qlo, qhi, blo, bhi, t);
            const bool da = la && ca < n - 1, db = lb && cb < n - 1;  // internal children to descend
            if (la && !da) emit_leaf<FILL>(D, i, ca - (n - 1), t, cnt, out);
            if (lb && !db) emit_leaf<FILL>(D, i, cb - (n - 1), t, cnt, out);
            if (da && db) {
                if (sp >= kStack) {
                    atomicOr(D.status, XPBD_STATUS_STACK_OVERFLOW);
                    break;
                }
                stack[sp++] = cb;
                node = ca;
            } else if (da || db) {
                node = da ? ca : cb;
            } else {
                if (sp == 0) break;
                node = stack[--sp];
            }
        }
    }
    if (!FILL) D.ws_count[t] = cnt;
}

__global__ void k_pairs_total(XpbdDcd D) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        const int tot = *D.ws_total;
        *D.n_pairs = tot;
        if (tot > D.max_pairs) atomicOr(D.status, XPBD_STATUS_PAIR_OVERFLOW);
        *D.n_contacts = 0;
    }
}

// ------------------------------------------------------------ narrowphase
__device__ __forceinline__ float3 pick3(float3 a, float3 b, float3 c, int i) { return i == 0 ? a : (i == 1 ? b : c); }

__device__ __forceinline__ bool inside_tri(float3 p1, float3 p2, float3 p3, float3 p) {
    const float3 c1 = cross(p2 - p1, p - p2), c2 = cross(p3 - p2, p - p3), c3 = cross(p1 - p3, p - p1);
    return dot(c1, c2) > 0.f && dot(c1, c3) > 0.f;
}

__device__ __forceinline__ float3 bary(float3 A, float3 B, float3 Cc, float3 P) {
    const float3 v0 = B - A, v1 = Cc - A, v2 = P - A;
    const float d00 = dot(v0, v0), d01 = dot(v0, v1), d11 = dot(v1, v1), d20 = dot(v2, v0), d21 = dot(v2, v1);
    const float den = d00 * d11 - d01 * d01;
    if (den == 0.f) return make_float3(1.f / 3.f, 1.f / 3.f, 1.f / 3.f);
    const float v = (d11 * d20 - d01 * d21) / den, w = (d00 * d21 - d01 * d20) / den;
    return make_float3(1.f - v - w, v, w);
}

__device__ __forceinline__ bool line_isect(float3 p1, float3 p2, float3 p3, float3 p4, float3 v1, float3 v2,
                                           float3& out) {
    const float3 d1 = p2 - p1, d2 = p4 - p3;
    const float3 nrm = cross(d1, d2);
    if (len(nrm) < 1.0e-6f) return false;
    const float den = dot(nrm, nrm);
    if (den < 1.0e-6f) return false;
    const float3 v = p3 - p1;
    const float t1 = dot(cross(v, d2), nrm) / den, t2 = dot(cross(v, d1), nrm) / den;
    if (!(t2 >= 0.f && t2 <= 1.f && t1 >= 0.f && t1 <= 1.f)) return false;
    out = v1 + t1 * (v2 - v1);
    return true;
}

__device__ __forceinline__ bool gen_t(float3 N, float3 v0, float3 v1, float3 v2, float d, float3 D, float2& iv) {
    const float d0 = dot(N, v0) + d, d1 = dot(N, v1) + d, d2 = dot(N, v2) + d;
    if (d0 <= kThresh && d1 <= kThresh && d2 <= kThresh) return false;
    if (d0 >= -kThresh && d1 >= -kThresh && d2 >= -kThresh) return false;
    float3 s0 = v0, s1 = v1, s2 = v2;
    float e0 = d0, e1 = d1, e2 = d2;
    if ((d0 <= 0.f && d1 >= 0.f && d2 >= 0.f) || (d0 >= 0.f && d1 <= 0.f && d2 <= 0.f)) {
        s0 = v1; s1 = v0; e0 = d1; e1 = d0;
    } else if ((d0 >= 0.f && d1 >= 0.f && d2 <= 0.f) || (d0 <= 0.f && d1 <= 0.f && d2 >= 0.f)) {
        s1 = v2; s2 = v1; e1 = d2; e2 = d1;
    }
    const float p0 = dot(D, s0), p1 = dot(D, s1), p2 = dot(D, s2);
    const float tA = p0 + (p1 - p0) * fabsf(e0 / (e0 - e1));
    const float tB = p2 + (p1 - p2) * fabsf(e2 / (e2 - e1));
    iv = tA > tB ? make_float2(tB, tA) : make_float2(tA, tB);
    return true;
}

__global__ void k_narrow(XpbdDcd D, const float* __restrict__ pos4) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int np = min(*D.n_pairs, D.max_pairs);
    if (k >= np) return;
    const int ta = D.pairs[2 * k], tb = D.pairs[2 * k + 1];
    const float3 q00 = f3(ld4(pos4, D.tris[3 * ta])), q01 = f3(ld4(pos4, D.tris[3 * ta + 1])),
                 q02 = f3(ld4(pos4, D.tris[3 * ta + 2]));
    const float3 q10 = f3(ld4(pos4, D.tris[3 * tb])), q11 = f3(ld4(pos4, D.tris[3 * tb + 1])),
                 q12 = f3(ld4(pos4, D.tris[3 * tb + 2]));
    const float3 n1f = cross(q01 - q00, q02 - q00), n2f = cross(q11 - q10, q12 - q10);
    const float l1 = len(n1f), l2 = len(n2f);
    if (l1 == 0.f || l2 == 0.f) return;
    const float3 N1 = n1f / l1, N2 = n2f / l2;
    const float d1 = -dot(N1, q00), d2 = -dot(N2, q10);
    const float3 cp = cross(N1, N2);
    const float lcp = len(cp);
    if (lcp < 1.0e-8f) return;
    const float3 Dd = cp / lcp;
    float2 iv1, iv2;
    if (!gen_t(N2, q00, q01, q02, d2, Dd, iv1)) return;
    if (!gen_t(N1, q10, q11, q12, d1, Dd, iv2)) return;
    if (!(iv1.y >= iv2.x && iv2.y >= iv1.x)) return;
    float C1 = 0.f, C2 = 0.f;
    float3 b1 = make_float3(0.f, 0.f, 0.f), b2 = b1, b3 = b1, b4 = b1;
    for (int j = 0; j < 3; ++j) {
        const float3 q0j = pick3(q00, q01, q02, j), q1j = pick3(q10, q11, q12, j);
        const float3 P0j = q0j - dot(N2, q0j - q10) * N2;
        if (inside_tri(q10, q11, q12, P0j)) {
            const float cand = dot(N2, q0j) + d2;
            if (C1 < -cand) {
                C1 = -cand;
                b1 = bary(q00, q01, q02, q0j);
                b2 = bary(q10, q11, q12, q0j - cand * N2);
            }
        }
        {
            const float den = dot(N1, N2);
            if (den != 0.f) {
                const float t = dot(N1, q00 - q1j) / den;
                const float3 Q0j = q1j + t * N2;
                if (inside_tri(q00, q01, q02, Q0j)) {
                    const float cand = dot(N2, Q0j) + d2;
                    if (C1 < -cand) {
                        C1 = -cand;
                        b1 = bary(q00, q01, q02, Q0j);
                        b2 = bary(q10, q11, q12, Q0j - cand * N2);
                    }
                }
            }
        }
        const float3 P1j = q1j - dot(N1, q1j - q00) * N1;
        if (inside_tri(q00, q01, q02, P1j)) {
            const float cand = dot(N1, q1j) + d1;
            if (C2 < -cand) {
                C2 = -cand;
                b3 = bary(q10, q11, q12, q1j);
                b4 = bary(q00, q01, q02, q1j - cand * N1);
            }
        }
        {
            const float den = dot(N2, N1);
            if (den != 0.f) {
                const float t = dot(N2, q10 - q0j) / den;
                const float3 Q1j = q0j + t * N1;
                if (inside_tri(q10, q11, q12, Q1j)) {
                    const float cand = dot(N1, Q1j) + d1;
                    if (C2 < -cand) {
                        C2 = -cand;
                        b3 = bary(q10, q11, q12, Q1j);
                        b4 = bary(q00, q01, q02, Q1j - cand * N1);
                    }
                }
            }
        }
        const int jn = (j + 1) % 3;
        const float3 q0jn = pick3(q00, q01, q02, jn), q1jn = pick3(q10, q11, q12, jn);
        const float3 P0jn = q0jn - dot(N2, q0jn - q10) * N2;
        const float3 P1jn = q1jn - dot(N1, q1jn - q00) * N1;
        for (int kk = 0; kk < 3; ++kk) {
            const int kn = (kk + 1) % 3;
            float3 o;
            if (line_isect(P0j, P0jn, pick3(q10, q11, q12, kk), pick3(q10, q11, q12, kn), q0j, q0jn, o)) {
                const float cand = dot(N2, o) + d2;
                if (C1 < -cand) {
                    C1 = -cand;
                    b1 = bary(q00, q01, q02, o);
                    b2 = bary(q10, q11, q12, o - cand * N2);
                }
            }
            if (line_isect(P1j, P1jn, pick3(q00, q01, q02, kk), pick3(q00, q01, q02, kn), q1j, q1jn, o)) {
                const float cand = dot(N1, o) + d1;
                if (C2 < -cand) {
                    C2 = -cand;
                    b3 = bary(q10, q11, q12, o);
                    b4 = bary(q00, q01, q02, o - cand * N1);
                }
            }
        }
    }
    if (C1 <= D.offset_eps || C2 <= D.offset_eps) return;
    const int slot = atomicAdd(D.n_contacts, 1);
    if (slot >= D.max_contacts) {
        atomicOr(D.status, XPBD_STATUS_CONTACT_OVERFLOW);
        return;
    }
    const bool first = C1 < C2;  // tie -> C2 branch
    const int tc = first ? ta : tb, tl = first ? tb : ta;
    int4* cid = reinterpret_cast<int4*>(D.c_ids);
    cid[2 * slot] = make_int4(D.tris[3 * tc], D.tris[3 * tc + 1], D.tris[3 * tc + 2], k);
    cid[2 * slot + 1] = make_int4(D.tris[3 * tl], D.tris[3 * tl + 1], D.tris[3 * tl + 2], 0);
    float4* cf = reinterpret_cast<float4*>(D.c_data);
    const float3 n = first ? N2 : N1;
    const float3 bb1 = first ? b1 : b3, bb2 = first ? b2 : b4;
    cf[3 * slot] = make_float4(n.x, n.y, n.z, first ? C1 : C2);
    cf[3 * slot + 1] = make_float4(bb1.x, bb1.y, bb1.z, C1);
    cf[3 * slot + 2] = make_float4(bb2.x, bb2.y, bb2.z, C2);
}

// respond_kernel (udcf/kernel.py:713-806)
__global__ void k_respond(XpbdDcd D, const float* __restrict__ pos4) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int nc = min(*D.n_contacts, D.max_contacts);
    if (k >= nc) return;
    const int4 cu = reinterpret_cast<const int4*>(D.c_ids)[2 * k];
    const int4 cl = reinterpret_cast<const int4*>(D.c_ids)[2 * k + 1];
    const float4 f0 = reinterpret_cast<const float4*>(D.c_data)[3 * k];
    const float4 f1 = reinterpret_cast<const float4*>(D.c_data)[3 * k + 1];
    const float4 f2 = reinterpret_cast<const float4*>(D.c_data)[3 * k + 2];
    float pen = f0.w;
    if (D.max_push > 0.f && pen > D.max_push) pen = D.max_push;
    float C = pen * D.multiplier;
    if (C == 0.f) return;
    const float3 nrm = make_float3(f0.x, f0.y, f0.z);
    const float4 pu0 = ld4(pos4, cu.x), pu1 = ld4(pos4, cu.y), pu2 = ld4(pos4, cu.z);
    const float4 pl0 = ld4(pos4, cl.x), pl1 = ld4(pos4, cl.y), pl2 = ld4(pos4, cl.z);
    const bool solid_cur = pu0.w == 0.f || pu1.w == 0.f || pu2.w == 0.f;
    const bool solid_clo = pl0.w == 0.f || pl1.w == 0.f || pl2.w == 0.f;
    if (!solid_cur && !solid_clo) C = C * 0.5f;
    const float3 push_clo = solid_clo ? make_float3(0.f, 0.f, 0.f) : (-C) * nrm;
    const float3 push_cur = solid_cur ? make_float3(0.f, 0.f, 0.f) : C * nrm;
    const float4* xp = reinterpret_cast<const float4*>(D.x_prev);
    const float3 v0 = (f3(pl0) + push_clo) - f3(xp[cl.x]), v1 = (f3(pl1) + push_clo) - f3(xp[cl.y]),
                 v2 = (f3(pl2) + push_clo) - f3(xp[cl.z]);
    const float3 v3 = (f3(pu0) + push_cur) - f3(xp[cu.x]), v4 = (f3(pu1) + push_cur) - f3(xp[cu.y]),
                 v5 = (f3(pu2) + push_cur) - f3(xp[cu.z]);
    const float3 g = nrm / len(nrm);
    const float3 b1 = make_float3(f1.x, f1.y, f1.z), b2 = make_float3(f2.x, f2.y, f2.z);
    const float3 vclo = (b1.x * v0 + b1.y * v1) + b1.z * v2;
    const float3 perp_clo = vclo - dot(vclo, g) * g;
    const float3 vcur = (b2.x * v3 + b2.y * v4) + b2.z * v5;
    const float3 perp_cur = vcur - dot(vcur, g) * g;
    float3 diff = perp_cur - perp_clo;
    const float dn = len(diff);
    const float static_norm = pen * D.friction_static;
    if (dn > static_norm && dn > 0.f) diff = (pen * D.friction_dynamic / dn) * diff;
    const float3 diffV = 0.5f * diff;
    const float3 diffT = diff - diffV;
    float4* acc = reinterpret_cast<float4*>(D.dP);
    const float3 mu = push_cur - diffV, ml = push_clo + diffT;
    if (pu0.w > 0.f) atomicAdd(&acc[cu.x], make_float4(mu.x, mu.y, mu.z, 1.f));
    if (pu1.w > 0.f) atomicAdd(&acc[cu.y], make_float4(mu.x, mu.y, mu.z, 1.f));
    if (pu2.w > 0.f) atomicAdd(&acc[cu.z], make_float4(mu.x, mu.y, mu.z, 1.f));
    if (pl0.w > 0.f) atomicAdd(&acc[cl.x], make_float4(ml.x, ml.y, ml.z, 1.f));
    if (pl1.w > 0.f) atomicAdd(&acc[cl.y], make_float4(ml.x, ml.y, ml.z, 1.f));
    if (pl2.w > 0.f) atomicAdd(&acc[cl.z], make_float4(ml.x, ml.y, ml.z, 1.f));
}

// apply_kernel (udcf/kernel.py:809-822), clearing the accumulator it reads
__global__ void k_dcd_apply(XpbdDcd D, float* pos4) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.n_verts) return;
    float4* acc = reinterpret_cast<float4*>(D.dP);
    const float4 a = acc[i];
    if (a.w > 0.f) {
        float4 p = reinterpret_cast<float4*>(pos4)[i];
        if (D.jacobi_avg) {
            p.x += a.x / a.w;
            p.y += a.y / a.w;
            p.z += a.z / a.w;
        } else {
            p.x += a.x;
            p.y += a.y;
            p.z += a.z;
        }
        reinterpret_cast<float4*>(pos4)[i] = p;
        acc[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
}

__global__ void k_copy4(const float4* __restrict__ src, float4* __restrict__ dst, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[i];
}

// Sort CTAs: one per kSortThreads keys, at most the co-resident count.
int64_t hist_words(int n) { return int64_t(256) * ((n + kSortThreads - 1) / kSortThreads); }
int64_t scan_words(int n) { return (n + kScanBlock - 1) / kScanBlock; }

int launch_sort(const XpbdDcd* D, uint32_t* sync, cudaStream_t s) {
    static int slots[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return cuda_check("xpbd_dcd_broadphase: device");
    if (slots[dev] == 0) {
        int n_sm = 0, per_sm = 0;
        if (cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sort_coop, kSortThreads, 0) != cudaSuccess)
            return cuda_check("xpbd_dcd_broadphase: sort occupancy");
        if (per_sm < 1) return fail(XPBD_ERR_LIMIT, "xpbd_dcd_broadphase: sort kernel does not fit an SM");
        slots[dev] = per_sm * n_sm;
    }
    const int n = D->n_tris;
    const int need = (n + kSortThreads - 1) / kSortThreads;
    const int G = std::min(need, slots[dev]);
    const int chunk = ((n + G - 1) / G + kSortThreads - 1) / kSortThreads * kSortThreads;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(G);
    cfg.blockDim = dim3(kSortThreads);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (cudaLaunchKernelEx(&cfg, k_sort_coop, *D, chunk, sync) != cudaSuccess)
        return cuda_check("xpbd_dcd_broadphase: sort launch");
    return XPBD_OK;
}

int check_dcd(const XpbdDcd* D) {
    if (!D || D->n_tris <= 0 || D->n_verts <= 0 || !D->tris || !D->pairs || !D->n_pairs || !D->n_contacts ||
        !D->c_ids || !D->c_data || !D->x_prev || !D->dP || !D->status || !D->ws_nodes || !D->ws_keys || !D->ws_vals ||
        !D->ws_keys2 || !D->ws_vals2 || !D->ws_hist || !D->ws_bbox || !D->ws_split || !D->ws_count ||
        !D->ws_total || !D->ws_slots)
        return fail(XPBD_ERR_ARG, "XpbdDcd: null member or empty size");
    if (D->max_pairs <= 0 || D->max_contacts <= 0) return fail(XPBD_ERR_ARG, "XpbdDcd: capacities must be > 0");
    if (!aligned16(D->ws_nodes) || !aligned16(D->ws_bbox) || !aligned16(D->ws_split) || !aligned16(D->pairs) || !aligned16(D->c_ids) || !aligned16(D->c_data) || !aligned16(D->x_prev) ||
        !aligned16(D->dP))
        return fail(XPBD_ERR_ALIGN, "XpbdDcd: 16-byte alignment");
    return XPBD_OK;
}

}  // namespace

extern "C" {

int xpbd_dcd_workspace_query(int32_t n_tris, XpbdDcdWorkspaceSizes* out) {
    if (n_tris <= 0 || !out) return fail(XPBD_ERR_ARG, "xpbd_dcd_workspace_query: bad arguments");
    out->nodes_floats = (tri_leaf_base(n_tris) + 2 * int64_t(n_tris)) * 4;  // records, leaves x2
    out->keys = n_tris;
    // sort histograms [CTAs][256], the count scan's block sums, the sort's barrier words
    out->hist = hist_words(n_tris) + scan_words(n_tris) + 4;
    out->bbox_floats = int64_t(8) * ((n_tris + 31) / 32 + (n_tris + 1023) / 1024);  // 32- and 1024-leaf block boxes
    out->count = n_tris;
    out->slots = int64_t(kSlots) * n_tris;
    out->split = int64_t(4) * (n_tris > 1 ? n_tris - 1 : 1);
    return XPBD_OK;
}

int xpbd_dcd_broadphase(const XpbdDcd* D, const float* pos4, int32_t snapshot_prev, xpbd_stream_t stream) {
    int rc;
    if ((rc = check_dcd(D))) return rc;
    if (!pos4 || !aligned16(pos4)) return fail(XPBD_ERR_ARG, "xpbd_dcd_broadphase: pos4");
    cudaStream_t s = (cudaStream_t)stream;
    const int n = D->n_tris;
    if (snapshot_prev)
        k_copy4<<<(D->n_verts + 255) / 256, 256, 0, s>>>(reinterpret_cast<const float4*>(pos4),
                                                          reinterpret_cast<float4*>(D->x_prev), D->n_verts);
    int* scan_scratch = D->ws_hist + hist_words(n);
    if (D->refit_only) {
        k_tri_aabb<false><<<(n + 255) / 256, 256, 0, s>>>(*D, pos4);
        k_permute_leaves<<<(n + 1023) / 1024, 1024, 0, s>>>(*D);
        if (n > 1) k_refit_ranges<<<(2 * (n - 1) + 255) / 256, 256, 0, s>>>(*D);
    } else {
        k_tri_aabb<true><<<(n + 255) / 256, 256, 0, s>>>(*D, pos4);
        uint32_t* sort_sync = reinterpret_cast<uint32_t*>(scan_scratch + scan_words(n));
        if ((rc = launch_sort(D, sort_sync, s))) return rc;
        k_permute_leaves<<<(n + 1023) / 1024, 1024, 0, s>>>(*D);
        if (n > 1) k_build<<<(2 * (n - 1) + 255) / 256, 256, 0, s>>>(*D);
    }
    k_traverse<false><<<(n + 127) / 128, 128, 0, s>>>(*D);
    scan_excl(D->ws_count, n, D->ws_total, scan_scratch, s);
    k_traverse<true><<<(n + 127) / 128, 128, 0, s>>>(*D);
    k_pairs_total<<<1, 32, 0, s>>>(*D);
    return cuda_check("xpbd_dcd_broadphase");
}

int xpbd_dcd_narrow_respond(const XpbdDcd* D, float* pos4, xpbd_stream_t stream) {
    int rc;
    if ((rc = check_dcd(D))) return rc;
    if (!pos4 || !aligned16(pos4)) return fail(XPBD_ERR_ARG, "xpbd_dcd_narrow_respond: pos4");
    cudaStream_t s = (cudaStream_t)stream;
    cudaMemsetAsync(D->n_contacts, 0, sizeof(int32_t), s);
    k_narrow<<<(D->max_pairs + 255) / 256, 256, 0, s>>>(*D, pos4);
    k_respond<<<(D->max_contacts + 255) / 256, 256, 0, s>>>(*D, pos4);
    k_dcd_apply<<<(D->n_verts + 255) / 256, 256, 0, s>>>(*D, pos4);
    return cuda_check("xpbd_dcd_narrow_respond");
}

}  // extern "C"
