// trace_plain.cu - the plain form: megakernels that reproduce the reference's
// compute-only shader (shaders/ray_trace.comp.hybrid.hlsl) operation for
// operation, one thread per ray or per pixel.  This is the parity baseline the
// optimised kernels are measured against.
#include "kernels.h"
#include "shade.cuh"
#include "trace_common.cuh"

namespace ae {

// ---------------------------------------------------------------------------
// Closest hit over a ray batch
// ---------------------------------------------------------------------------
// WT: the watertight triangle test in the same walk (AE_VARIANT_PLAIN_WT).
template <bool WT>
__global__ void __launch_bounds__(128) k_closest_plain(DevScene S, const ae_ray *__restrict__ rays, uint32_t n,
                                                       ae_hit *__restrict__ hits) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 *rp = reinterpret_cast<const float4 *>(rays + i);
    const float4 r0 = __ldg(rp), r1 = __ldg(rp + 1);
    uint32_t seed = 1u;
    DHit h;
    ae_hit out;
    out.t = 0.0f; out.alpha = 0.0f; out.beta = 0.0f; out.object = AE_MISS; out.prim = AE_MISS;
    if (traverse_ref<WT>(S, mk(r0.x, r0.y, r0.z), mk(r1.x, r1.y, r1.z), r1.w, r0.w, h, seed)) {
        out.t = h.t; out.alpha = h.alpha; out.beta = h.beta; out.object = h.slot; out.prim = h.prim;
    }
    hits[i] = out;
}

// The debug walk (AE_VARIANT_PLAIN_CHECKED): PLAIN's traversal with every
// stack push and buffer index checked (Checks).
__global__ void __launch_bounds__(128) k_closest_checked(DevScene S, Checks C, const ae_ray *__restrict__ rays,
                                                         uint32_t n, ae_hit *__restrict__ hits) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 *rp = reinterpret_cast<const float4 *>(rays + i);
    const float4 r0 = __ldg(rp), r1 = __ldg(rp + 1);
    uint32_t seed = 1u;
    DHit h;
    ae_hit out;
    out.t = 0.0f; out.alpha = 0.0f; out.beta = 0.0f; out.object = AE_MISS; out.prim = AE_MISS;
    if (traverse_ref<false>(S, mk(r0.x, r0.y, r0.z), mk(r1.x, r1.y, r1.z), r1.w, r0.w, h, seed, nullptr, &C)) {
        out.t = h.t; out.alpha = h.alpha; out.beta = h.beta; out.object = h.slot; out.prim = h.prim;
    }
    hits[i] = out;
}

cudaError_t launch_closest_checked(const DevScene &S, const Checks &C, const ae_ray *rays, uint32_t n, ae_hit *hits,
                                   cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    k_closest_checked<<<(n + 127) / 128, 128, 0, st>>>(S, C, rays, n, hits);
    return cudaGetLastError();
}

// The same traversal with its touches counted: the algorithmic traffic of
// the reference's walk, per ray set, summed in 64-bit.
__global__ void __launch_bounds__(128) k_count_plain(DevScene S, const ae_ray *__restrict__ rays, uint32_t n,
                                                     unsigned long long *__restrict__ totals) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    Touch T = {0, 0, 0, 0, 0, 0, 0};
    if (i < n) {
        const float4 *rp = reinterpret_cast<const float4 *>(rays + i);
        const float4 r0 = __ldg(rp), r1 = __ldg(rp + 1);
        uint32_t seed = 1u;
        DHit h;
        traverse_ref(S, mk(r0.x, r0.y, r0.z), mk(r1.x, r1.y, r1.z), r1.w, r0.w, h, seed, &T);
    }
    const uint32_t v[6] = {T.tlas, T.objects, T.instances, T.blas, T.tris, T.winners};
    for (int k = 0; k < 6; k++) {
        unsigned long long x = v[k];
        for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
        if ((threadIdx.x & 31) == 0 && x) atomicAdd(totals + k, x);
    }
}

// ---------------------------------------------------------------------------
// Compute-only path tracer (hybrid:1230-1404)
// ---------------------------------------------------------------------------
// ColorRay, hybrid:1230-1325.  T (optional) counts every traversal's touches.
AE_DEV f3 color_ray(const DevScene &S, const FrameParams &F, f3 o, f3 d, float time, uint32_t &seed,
                    Touch *T = nullptr) {
    f3 thr = splat(1.0f), acc = splat(0.0f);
    for (uint32_t b = 0; b < F.depth; b++) {
        DHit h;
        if (!traverse_ref(S, o, d, time, 0.001f, h, seed, T)) {
            acc = acc + thr * F.sky;
            break;
        }
        const MatRec m = load_mat(S.objects + h.slot);
        if (m.type == AE_MAT_DIFFUSE_LIGHT) {
            acc = acc + thr * (m.emission * m.albedo);
            break;
        }
        // SurfaceAlbedo (textured when the material has a layer).
        const f3 alb = m.type != AE_MAT_DIELECTRIC ? surface_albedo(S, h, m, o, d) : m.albedo;
        if (m.type == AE_MAT_LAMBERTIAN) {
            f3 dl = direct_light(S, h, alb, time, seed, T);
            const float luma = maxc(dl);
            if (luma > 8.0f) dl = dl * AE_DIV(8.0f, luma);
            acc = acc + thr * dl;
        }
        f3 sd, gw;
        if (!get_bounce(d, h, m, alb, sd, gw, seed)) break;
        d = normalize(sd);
        const float sgn = dot(d, h.n) < 0.0f ? -1.0f : 1.0f;
        o = h.p + h.n * AE_MUL(0.001f, sgn);
        if (m.type == AE_MAT_GGX_METAL) thr = thr * gw;
        else if (m.type != AE_MAT_DIELECTRIC) thr = thr * alb;
        if (b > 0) {
            const float p = clampf(maxc(thr), 0.1f, 1.0f);
            if (rng_next(seed) > p) break;
            thr = thr / p;
        }
    }
    return acc;
}

// main, hybrid:1328-1404.  Threads cover 16x8 pixel tiles so a warp's rays
// start coherent; the result per pixel does not depend on the mapping.
__global__ void __launch_bounds__(128) k_render_plain(DevScene S, FrameParams F, float4 *__restrict__ accum,
                                                      uchar4 *__restrict__ display, float4 *__restrict__ frame) {
    const uint32_t x = blockIdx.x * 16 + (threadIdx.x & 15);
    const uint32_t y = blockIdx.y * 8 + (threadIdx.x >> 4);
    if (x >= F.width || y >= F.height) return;
    const size_t px = size_t(y) * F.width + x;
    if (F.display_only) {
        const float4 a = accum[px];
        display[px] = display_texel(mk(a.x, a.y, a.z), F.exposure);
        return;
    }
    uint32_t seed = x + y * F.width + F.batch * F.width * F.height + 1u;
    f3 color = splat(0.0f);
    for (uint32_t s = 0; s < F.spp; s++) {
        const float jx = AE_SUB(rng_next(seed), 0.5f);
        const float jy = AE_SUB(rng_next(seed), 0.5f);
        const f3 tgt = F.pixel0 + AE_ADD(AE_U2F(x), jx) * F.pixel_u + AE_ADD(AE_U2F(y), jy) * F.pixel_v;
        f3 o = F.source;
        if (F.defocus_angle > 0.0f) {
            float px_, py_;
            for (;;) {
                const float a = rng_next(seed), b = rng_next(seed);
                px_ = AE_SUB(AE_MUL(a, 2.0f), 1.0f);
                py_ = AE_SUB(AE_MUL(b, 2.0f), 1.0f);
                if (length(mk(px_, py_, 0.0f)) < 1.0f) break;
            }
            o = F.source + px_ * F.defocus_u + py_ * F.defocus_v;
        }
        const f3 d = normalize(tgt - o);
        const float time = rng_next(seed);
        color = color + color_ray(S, F, o, d, time, seed);
    }
    color = color / AE_U2F(F.spp);
    if (frame) frame[px] = make_float4(color.x, color.y, color.z, 1.0f);
    f3 acc;
    if (F.batch == 0) {
        acc = color;
    } else {
        const float4 prev = accum[px];
        const float w = AE_DIV(1.0f, AE_U2F(F.batch + 1));
        acc = lerp(mk(prev.x, prev.y, prev.z), color, w);
    }
    accum[px] = make_float4(acc.x, acc.y, acc.z, 1.0f);
    display[px] = display_texel(acc, F.exposure);
}

// The frame's paths (main's camera ray and ColorRay, spp samples per pixel)
// with every traversal's touches counted - the algorithmic traffic per path
// of the reference's megakernel.  Writes no image; outside timed regions.
__global__ void __launch_bounds__(128) k_count_paths(DevScene S, FrameParams F,
                                                     unsigned long long *__restrict__ totals) {
    const uint32_t x = blockIdx.x * 16 + (threadIdx.x & 15);
    const uint32_t y = blockIdx.y * 8 + (threadIdx.x >> 4);
    Touch T = {0, 0, 0, 0, 0, 0, 0};
    if (x < F.width && y < F.height) {
        uint32_t seed = x + y * F.width + F.batch * F.width * F.height + 1u;
        for (uint32_t s = 0; s < F.spp; s++) {
            const float jx = AE_SUB(rng_next(seed), 0.5f);
            const float jy = AE_SUB(rng_next(seed), 0.5f);
            const f3 tgt = F.pixel0 + AE_ADD(AE_U2F(x), jx) * F.pixel_u + AE_ADD(AE_U2F(y), jy) * F.pixel_v;
            f3 o = F.source;
            if (F.defocus_angle > 0.0f) {
                float px_, py_;
                for (;;) {
                    const float a = rng_next(seed), b = rng_next(seed);
                    px_ = AE_SUB(AE_MUL(a, 2.0f), 1.0f);
                    py_ = AE_SUB(AE_MUL(b, 2.0f), 1.0f);
                    if (length(mk(px_, py_, 0.0f)) < 1.0f) break;
                }
                o = F.source + px_ * F.defocus_u + py_ * F.defocus_v;
            }
            const f3 d = normalize(tgt - o);
            const float time = rng_next(seed);
            color_ray(S, F, o, d, time, seed, &T);
        }
    }
    const uint32_t v[7] = {T.tlas, T.objects, T.instances, T.blas, T.tris, T.winners, T.rays};
    for (int k = 0; k < 7; k++) {
        unsigned long long c = v[k];
        for (int off = 16; off > 0; off >>= 1) c += __shfl_down_sync(0xffffffffu, c, off);
        if ((threadIdx.x & 31) == 0 && c) atomicAdd(totals + k, c);
    }
}

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------
cudaError_t launch_closest_plain(const DevScene &S, const ae_ray *rays, uint32_t n, ae_hit *hits, cudaStream_t st,
                                 bool watertight) {
    if (n == 0) return cudaSuccess;
    if (watertight) k_closest_plain<true><<<(n + 127) / 128, 128, 0, st>>>(S, rays, n, hits);
    else k_closest_plain<false><<<(n + 127) / 128, 128, 0, st>>>(S, rays, n, hits);
    return cudaGetLastError();
}

cudaError_t launch_count_plain(const DevScene &S, const ae_ray *rays, uint32_t n, unsigned long long *totals,
                               cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    k_count_plain<<<(n + 127) / 128, 128, 0, st>>>(S, rays, n, totals);
    return cudaGetLastError();
}

cudaError_t launch_count_paths(const DevScene &S, const FrameParams &F, unsigned long long *totals, cudaStream_t st) {
    dim3 grid((F.width + 15) / 16, (F.height + 7) / 8);
    k_count_paths<<<grid, 128, 0, st>>>(S, F, totals);
    return cudaGetLastError();
}

cudaError_t launch_render_plain(const DevScene &S, const FrameParams &F, float4 *accum, uchar4 *display, float4 *frame,
                                cudaStream_t st) {
    dim3 grid((F.width + 15) / 16, (F.height + 7) / 8);
    k_render_plain<<<grid, 128, 0, st>>>(S, F, accum, display, frame);
    return cudaGetLastError();
}

}  // namespace ae
