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
bool g_accum_dirty[kMaxDevices] = {};
std::mutex g_setup_mutex;

// Device address of g_noalloc_accum on the current device.  In host code the
// symbol's name is only a host-side handle, so the address must come from
// cudaGetSymbolAddress with that device current.  It is looked up again on
// every call made outside stream capture, so a module reloaded after a device
// reset is picked up; a call made while `s` is being captured uses the address
// of the last uncaptured call on the device and fails when there was none.
int accum_address(cudaStream_t s, float4** out, int* dev_out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return xpbd::cuda_check("xpbd_iterate_noalloc: cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) return xpbd::fail(XPBD_ERR_LIMIT, "xpbd_iterate_noalloc: device index too large");
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cap) != cudaSuccess) return xpbd::cuda_check("xpbd_iterate_noalloc: capture query");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (cap == cudaStreamCaptureStatusNone) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_accum);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return xpbd::fail(XPBD_ERR_CUDA, "xpbd_iterate_noalloc: cudaGetSymbolAddress failed");
        }
        // a new module instance starts zeroed, like the first one
        if (static_cast<float4*>(p) != g_accum_ptr[dev]) g_accum_dirty[dev] = false;
        g_accum_ptr[dev] = static_cast<float4*>(p);
    } else if (!g_accum_ptr[dev]) {
        return xpbd::fail(XPBD_ERR_ARG,
                          "xpbd_iterate_noalloc: the first call on a device must come before any stream capture");
    }
    *out = g_accum_ptr[dev];
    *dev_out = dev;
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
    int dev = 0;
    cudaStream_t s = (cudaStream_t)stream;
    int rc = accum_address(s, &acc, &dev);
    if (rc) return rc;
    // The iteration expects an all-zero accumulator and leaves it all zero
    // (interior vertices never touch it, APPLY_CLEAR zeroes the boundary
    // slots), and the array starts zeroed: it is cleared only after a call
    // that stopped between its two launches.
    if (g_accum_dirty[dev]) {
        if (cudaMemsetAsync(acc, 0, size_t(XPBD_NOALLOC_MAX_VERTS) * sizeof(float4), s) != cudaSuccess)
            return xpbd::cuda_check("xpbd_iterate_noalloc: clear");
        g_accum_dirty[dev] = false;
    }
    XpbdVerts w = *v;
    w.accum = reinterpret_cast<float*>(acc);
    g_accum_dirty[dev] = true;
    rc = xpbd_project(prm, tiles, &w, XPBD_PROJECT_FUSED, stream);
    if (rc) return rc;
    rc = xpbd_apply_boundary(prm, tiles, &w, XPBD_APPLY_ATTACH | XPBD_APPLY_DIVIDE | XPBD_APPLY_PIN | XPBD_APPLY_CLEAR,
                             stream);
    if (rc) return rc;
    g_accum_dirty[dev] = false;
    return XPBD_OK;
}
