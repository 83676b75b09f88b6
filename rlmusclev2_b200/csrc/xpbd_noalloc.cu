// Allocation-free variant of one Jacobi iteration.
//
// Some hosts cannot hand this library a scratch buffer or let it allocate one:
// a simulation step recorded inside another framework's CUDA graph capture
// (cudaMalloc is not a legal call while a stream is being captured), a plugin
// running in a process whose device memory is owned by another allocator (a
// game or rendering engine that reserves the GPU's memory up front), or a
// real-time loop that forbids allocation after start-up.  For them
// xpbd_iterate_noalloc runs the same fused iteration as xpbd_project
// (XPBD_PROJECT_FUSED) + xpbd_apply_boundary, but its Jacobi accumulator --
// the only scratch the iteration needs -- is a fixed array in this file's
// device memory instead of XpbdVerts.accum.
//
// The array holds XPBD_NOALLOC_MAX_VERTS float4 (4 MiB) and exists once per
// GPU that loads the library, until the process exits.  Every call shares it:
// calls whose GPU work overlaps (two streams, two threads) race on it and
// must be serialised by the caller.
#include <cuda_runtime.h>

#include <mutex>

#include "xpbd_common.cuh"

namespace {

static __device__ __align__(256) float4 g_noalloc_accum[XPBD_NOALLOC_MAX_VERTS];

constexpr int kMaxDevices = 64;
float4* g_accum_ptr[kMaxDevices] = {};
std::mutex g_setup_mutex;

// Device address of g_noalloc_accum on the current device.  In host code the
// symbol's name is only a host-side handle, so the address must come from
// cudaGetSymbolAddress, once per device, with that device current.
int accum_address(float4** out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return xpbd::cuda_check("xpbd_iterate_noalloc: cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) return xpbd::fail(XPBD_ERR_LIMIT, "xpbd_iterate_noalloc: device index too large");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_accum_ptr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_accum);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return xpbd::fail(XPBD_ERR_CUDA, "xpbd_iterate_noalloc: cudaGetSymbolAddress failed");
        }
        g_accum_ptr[dev] = static_cast<float4*>(p);
    }
    *out = g_accum_ptr[dev];
    return XPBD_OK;
}

}  // namespace

extern "C" int xpbd_iterate_noalloc(const XpbdParams* prm, const XpbdTiles* tiles, const XpbdVerts* v,
                                    xpbd_stream_t stream) {
    if (!prm || !tiles || !v) return xpbd::fail(XPBD_ERR_ARG, "xpbd_iterate_noalloc: null argument");
    if (v->n <= 0) return xpbd::fail(XPBD_ERR_ARG, "xpbd_iterate_noalloc: empty vertex set");
    if (v->n > XPBD_NOALLOC_MAX_VERTS)
        return xpbd::fail(XPBD_ERR_LIMIT, "xpbd_iterate_noalloc: more vertices than XPBD_NOALLOC_MAX_VERTS (262144)");
    float4* acc = nullptr;
    int rc = accum_address(&acc);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    // The iteration expects an all-zero accumulator; the array keeps whatever
    // the previous call left, so clear the range this mesh uses.
    if (cudaMemsetAsync(acc, 0, size_t(v->n) * sizeof(float4), s) != cudaSuccess)
        return xpbd::cuda_check("xpbd_iterate_noalloc: clear");
    XpbdVerts w = *v;
    w.accum = reinterpret_cast<float*>(acc);
    rc = xpbd_project(prm, tiles, &w, XPBD_PROJECT_FUSED, stream);
    if (rc) return rc;
    return xpbd_apply_boundary(prm, tiles, &w, XPBD_APPLY_ATTACH | XPBD_APPLY_DIVIDE | XPBD_APPLY_PIN | XPBD_APPLY_CLEAR,
                               stream);
}
