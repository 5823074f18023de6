// noalloc.cu - closest hit for host ray buffers without any device
// allocation.
//
// ae_closest_hit stages the caller's rays and hits in device buffers it
// allocates (and grows) on demand.  Some callers cannot let a library call
// cudaMalloc: a frame loop that must not stall on the device-wide
// synchronisation cudaMalloc and cudaFree imply, or a process whose device
// memory is already handed out by another allocator (a framework's caching
// pool), where a new allocation may fail or fragment the pool.  For them
// ae_closest_hit_noalloc stages through one fixed array compiled into the
// library, AE_NOALLOC_MAX_RAYS rays plus their hits (3.25 MiB), which every
// GPU that loads the library holds until the process exits.
//
// Rules of the shared array:
//   * host code may not use the array's name as a device address; the
//     address comes from cudaGetSymbolAddress, looked up once per device with
//     that device current, on the first call on that device.  That first
//     call should come before any stream capture;
//   * every call on a device reuses the same array and it keeps the last
//     call's contents.  Nothing in it needs to start at zero: each call
//     writes every ray and every hit it reads back.  Calls that overlap on
//     the GPU (two threads, or two contexts on one device) race on it;
//   * the cached address belongs to the device's primary context: after a
//     cudaDeviceReset (or anything else that destroys that context) it is
//     stale, so the entry point must not be used across a reset;
//   * the call makes the context's device current while it runs and gives
//     the calling thread back its previous current device on return.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "context.h"
#include "fast.h"
#include "fast_trace.cuh"
#include "kernels.h"

namespace {

constexpr uint32_t kMaxRays = AE_NOALLOC_MAX_RAYS;
constexpr size_t kRayBytes = size_t(kMaxRays) * sizeof(ae_ray);  // 2 MiB, a multiple of 256
constexpr size_t kHitBytes = size_t(kMaxRays) * sizeof(ae_hit);  // 1.25 MiB

static __device__ __align__(256) unsigned char g_noalloc_scratch[kRayBytes + kHitBytes];

constexpr int kMaxDevices = 64;
void *g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_lock;

}  // namespace

using namespace ae;

extern "C" int ae_closest_hit_noalloc(ae_ctx *ctx, const ae_ray *rays, uint32_t n, ae_hit *hits, int variant) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c) return AE_ERR_INVALID;
    if (n && (!rays || !hits)) return c->fail(AE_ERR_INVALID, "null ray or hit buffer");
    if (n > kMaxRays)
        return c->fail(AE_ERR_OVERSIZE, "ae_closest_hit_noalloc takes at most %u rays per call (got %u); split the batch",
                       kMaxRays, n);
    if (!c->scene_uploaded) return c->fail(AE_ERR_STATE, "trace before ae_upload_scene");
    if (variant == AE_VARIANT_FAST_WALK)
        return c->fail(AE_ERR_INVALID, "AE_VARIANT_FAST_WALK reserves per-launch counters in device memory the "
                                       "library allocates; use AE_VARIANT_FAST or AE_VARIANT_QUANT here");
    if (variant != AE_VARIANT_PLAIN && variant != AE_VARIANT_FAST && variant != AE_VARIANT_QUANT)
        return c->fail(AE_ERR_INVALID, "unknown kernel variant %d", variant);
    // The optimised structures are built (allocated) by ae_prepare_fast; this
    // entry point only uses them when they are current and were accepted for
    // this scene (the optimised kernels have no participating media).
    if (variant != AE_VARIANT_PLAIN) {
        if (!(c->fast_ready && c->fast && c->fast->scene_key == c->scene_version))
            return c->fail(AE_ERR_STATE, "call ae_prepare_fast (which allocates) before the no-allocation entry point");
        if (c->fast->has_volumes)
            return c->fail(AE_ERR_STATE, "participating media consume RNG in the reference's visit order; use the "
                                         "plain kernel");
    }
    const int dev = c->settings.device;
    if (dev < 0 || dev >= kMaxDevices) return c->fail(AE_ERR_INVALID, "device ordinal %d out of range", dev);
    int prev_dev = -1;
    if (cudaGetDevice(&prev_dev) != cudaSuccess) {
        cudaGetLastError();
        prev_dev = -1;
    }
    // Gives the calling thread its current device back on every return path.
    struct RestoreDevice {
        int dev;
        ~RestoreDevice() {
            if (dev >= 0) cudaSetDevice(dev);
        }
    } restore{prev_dev == dev ? -1 : prev_dev};
    int rc = c->cuda(cudaSetDevice(dev), "cudaSetDevice");
    if (rc) return rc;
    void *base;
    {
        std::lock_guard<std::mutex> guard(g_scratch_lock);
        if (!g_scratch_addr[dev]) {
            void *addr = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
            if (e != cudaSuccess || !addr) return c->cuda(e != cudaSuccess ? e : cudaErrorInvalidSymbol, "cudaGetSymbolAddress");
            g_scratch_addr[dev] = addr;
        }
        base = g_scratch_addr[dev];
    }
    if (n == 0) return AE_OK;
    ae_ray *d_rays = static_cast<ae_ray *>(base);
    ae_hit *d_hits = reinterpret_cast<ae_hit *>(static_cast<unsigned char *>(base) + kRayBytes);
    if ((rc = c->cuda(cudaMemcpyAsync(d_rays, rays, size_t(n) * sizeof(ae_ray), cudaMemcpyHostToDevice, c->stream),
                      "copy rays")))
        return rc;
    const cudaError_t le = variant == AE_VARIANT_PLAIN
                               ? launch_closest_plain(c->scene(), d_rays, n, d_hits, c->stream)
                               : launch_closest_fast(c, d_rays, n, d_hits, variant == AE_VARIANT_QUANT, c->stream);
    if ((rc = c->cuda(le, "closest hit launch"))) return rc;
    c->launches++;
    if ((rc = c->cuda(cudaMemcpyAsync(hits, d_hits, size_t(n) * sizeof(ae_hit), cudaMemcpyDeviceToHost, c->stream),
                      "copy hits")))
        return rc;
    return c->cuda(cudaStreamSynchronize(c->stream), "closest hit (no allocation)");
}
