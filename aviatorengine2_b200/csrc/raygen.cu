// raygen.cu - camera rays (main's per-pixel ray setup, hybrid:1346-1373) and
// one diffuse bounce from a closest hit (GetBounce's Lambertian rule,
// hybrid:980-986, origin offset hybrid:1294-1296), as standalone ray sets.
// These make the closest-hit workload: the primary set of a frame at Batch b
// and the incoherent bounce set that follows it.
#include "context.h"
#include "kernels.h"
#include "shade.cuh"
#include "trace_common.cuh"

namespace ae {

__global__ void k_camera_rays(FrameParams F, ae_ray *__restrict__ out) {
    const uint32_t x = blockIdx.x * 16 + (threadIdx.x & 15);
    const uint32_t y = blockIdx.y * 8 + (threadIdx.x >> 4);
    if (x >= F.width || y >= F.height) return;
    f3 o, d;
    float time;
    uint32_t seed;
    camera_ray(F, x, y, o, d, time, seed);
    float4 *p = reinterpret_cast<float4 *>(out + size_t(y) * F.width + x);
    p[0] = make_float4(o.x, o.y, o.z, 0.001f);
    p[1] = make_float4(d.x, d.y, d.z, time);
}

__global__ void k_bounce_rays(DevScene S, FrameParams F, const ae_ray *__restrict__ prim, const ae_hit *__restrict__ hits,
                              uint32_t n, ae_ray *__restrict__ out, uint8_t *__restrict__ valid) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const ae_ray r = prim[i];
    const ae_hit h = hits[i];
    const f3 o = mk(r.ox, r.oy, r.oz), d = mk(r.dx, r.dy, r.dz);
    f3 nrm;
    ae_ray b = r;
    uint8_t ok = 0;
    if (hit_normal(S, h, d, nrm)) {
        // The pixel's stream after its camera ray (pixel index i, row-major).
        f3 co, cd;
        float time;
        uint32_t seed;
        camera_ray(F, i % F.width, i / F.width, co, cd, time, seed);
        const float z = AE_SUB(AE_MUL(rng_next(seed), 2.0f), 1.0f);
        const float a = AE_MUL(rng_next(seed), 6.2831853f);
        const float rr = AE_SQRT(AE_SUB(1.0f, AE_MUL(z, z)));
        f3 dir = nrm + mk(AE_MUL(rr, cosf_(a)), AE_MUL(rr, sinf_(a)), z);
        if (dot(dir, dir) < 0.001f) dir = nrm;
        dir = normalize(dir);
        const f3 p = o + d * h.t;
        const float sgn = dot(dir, nrm) < 0.0f ? -1.0f : 1.0f;
        const f3 no = p + nrm * AE_MUL(0.001f, sgn);
        b.ox = no.x; b.oy = no.y; b.oz = no.z;
        b.dx = dir.x; b.dy = dir.y; b.dz = dir.z;
        b.tnear = 0.001f;
        ok = 1;
    }
    out[i] = b;
    valid[i] = ok;
}

}  // namespace ae

using namespace ae;

extern "C" int ae_camera_rays(ae_ctx *ctx, ae_ray *out) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c || !out) return AE_ERR_INVALID;
    const FrameParams F = make_frame_params(c->config);
    const size_t n = size_t(F.width) * F.height;
    DevBuf<ae_ray> d;
    if (d.reserve(n)) return c->fail(AE_ERR_OOM, "ray buffer");
    dim3 grid((F.width + 15) / 16, (F.height + 7) / 8);
    k_camera_rays<<<grid, 128, 0, c->stream>>>(F, d.ptr);
    c->launches++;
    int rc = c->cuda(cudaGetLastError(), "camera rays");
    if (!rc) rc = c->cuda(cudaMemcpyAsync(out, d.ptr, n * sizeof(ae_ray), cudaMemcpyDeviceToHost, c->stream), "copy");
    if (!rc) rc = c->cuda(cudaStreamSynchronize(c->stream), "camera rays");
    return rc;
}

extern "C" int ae_bounce_rays(ae_ctx *ctx, const ae_ray *prim, const ae_hit *hits, uint32_t n, ae_ray *out,
                              uint8_t *valid) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c || (n && (!prim || !hits || !out || !valid))) return AE_ERR_INVALID;
    if (!c->scene_uploaded) return c->fail(AE_ERR_STATE, "bounce rays before ae_upload_scene");
    const FrameParams F = make_frame_params(c->config);
    if (uint64_t(n) > uint64_t(F.width) * F.height)
        return c->fail(AE_ERR_INVALID, "bounce rays: %u rays exceed the %ux%u frame", n, F.width, F.height);
    // Hits must name existing objects and triangles before a kernel follows them.
    for (uint32_t i = 0; i < n; i++) {
        if (hits[i].object == AE_MISS) continue;
        if (hits[i].object >= c->n_objects) return c->fail(AE_ERR_LAYOUT, "hit %u names object %u", i, hits[i].object);
        const ae_object &o = c->host_objects[hits[i].object];
        if (o.shapeType == AE_SHAPE_MESH && hits[i].prim >= c->host_instances[o.instanceIndex].triangleCount)
            return c->fail(AE_ERR_LAYOUT, "hit %u names triangle %u", i, hits[i].prim);
    }
    if (n == 0) return AE_OK;
    DevBuf<ae_ray> dp, dout;
    DevBuf<ae_hit> dh;
    DevBuf<uint8_t> dv;
    if (dp.reserve(n) || dout.reserve(n) || dh.reserve(n) || dv.reserve(n)) return c->fail(AE_ERR_OOM, "bounce buffers");
    int rc = c->cuda(cudaMemcpyAsync(dp.ptr, prim, size_t(n) * sizeof(ae_ray), cudaMemcpyHostToDevice, c->stream), "copy");
    if (!rc) rc = c->cuda(cudaMemcpyAsync(dh.ptr, hits, size_t(n) * sizeof(ae_hit), cudaMemcpyHostToDevice, c->stream), "copy");
    if (rc) return rc;
    k_bounce_rays<<<(n + 127) / 128, 128, 0, c->stream>>>(c->scene(), F, dp.ptr, dh.ptr, n, dout.ptr, dv.ptr);
    c->launches++;
    rc = c->cuda(cudaGetLastError(), "bounce rays");
    if (!rc) rc = c->cuda(cudaMemcpyAsync(out, dout.ptr, size_t(n) * sizeof(ae_ray), cudaMemcpyDeviceToHost, c->stream), "copy");
    if (!rc) rc = c->cuda(cudaMemcpyAsync(valid, dv.ptr, n, cudaMemcpyDeviceToHost, c->stream), "copy");
    if (!rc) rc = c->cuda(cudaStreamSynchronize(c->stream), "bounce rays");
    return rc;
}
