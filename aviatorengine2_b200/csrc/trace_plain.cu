// trace_plain.cu - the plain form: megakernels that reproduce the reference's
// compute-only shader (shaders/ray_trace.comp.hybrid.hlsl) operation for
// operation, one thread per ray or per pixel.  This is the parity baseline the
// optimised kernels are measured against.
#include "kernels.h"
#include "trace_common.cuh"

namespace ae {

// ---------------------------------------------------------------------------
// Closest hit over a ray batch
// ---------------------------------------------------------------------------
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
    if (traverse_ref(S, mk(r0.x, r0.y, r0.z), mk(r1.x, r1.y, r1.z), r1.w, r0.w, h, seed)) {
        out.t = h.t; out.alpha = h.alpha; out.beta = h.beta; out.object = h.slot; out.prim = h.prim;
    }
    hits[i] = out;
}

// The same traversal with its touches counted: the algorithmic traffic of
// the reference's walk, per ray set, summed in 64-bit.
__global__ void __launch_bounds__(128) k_count_plain(DevScene S, const ae_ray *__restrict__ rays, uint32_t n,
                                                     unsigned long long *__restrict__ totals) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    Touch T = {0, 0, 0, 0, 0, 0};
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
struct MatRec {
    f3 albedo;
    float fuzz, emission, refraction;
    uint32_t type;
};
AE_DEV MatRec load_mat(const ae_object *o) {
    const char *b = reinterpret_cast<const char *>(o);
    const float4 m0 = ld4(b + 80), m1 = ld4(b + 96), m2 = ld4(b + 112);
    return MatRec{mk(m1.x, m1.y, m1.z), m1.w, m0.y, m2.x, __float_as_uint(m2.z)};
}

AE_DEV f3 random_direction(uint32_t &seed) {
    const float z = AE_SUB(AE_MUL(rng_next(seed), 2.0f), 1.0f);
    const float a = AE_MUL(rng_next(seed), 6.2831853f);
    const float r = AE_SQRT(AE_SUB(1.0f, AE_MUL(z, z)));
    return mk(AE_MUL(r, cosf_(a)), AE_MUL(r, sinf_(a)), z);
}

// SampleLight, hybrid:1057-1119.
AE_DEV void sample_light(const ae_object *L, uint32_t shape, f3 from, f3 &p, float &omega, uint32_t &seed) {
    const char *b = reinterpret_cast<const char *>(L);
    const float4 q0 = ld4(b);
    const f3 P = mk(q0.x, q0.y, q0.z);
    p = P;
    omega = 0.0f;
    if (shape == AE_SHAPE_QUAD) {
        const float4 q2 = ld4(b + 32), q3 = ld4(b + 48);
        const f3 U = mk(q2.x, q2.y, q2.z), W = mk(q3.x, q3.y, q3.z);
        const float r1 = rng_next(seed);
        const float r2 = rng_next(seed);
        p = P + r1 * U + r2 * W;
        const f3 cuv = cross(U, W);
        const float area = length(cuv);
        const f3 ln = cuv / fmax_(area, 1e-8f);
        f3 ts = from - p;
        const float d2 = dot(ts, ts);
        ts = normalize(ts);
        const float cl = AE_FABS(dot(ln, ts));
        omega = AE_DIV(AE_MUL(cl, area), fmax_(d2, 1e-8f));
        return;
    }
    if (shape == AE_SHAPE_SPHERE) {
        const float radius = ld4(b + 16).w;
        const f3 tl = P - from;
        const float d2 = fmax_(dot(tl, tl), 1e-8f);
        const float r2 = AE_MUL(radius, radius);
        if (d2 <= r2) { omega = AE_MUL(4.0f, 3.14159265f); return; }
        const float ctm = AE_SQRT(fmax_(0.0f, AE_SUB(1.0f, AE_DIV(r2, d2))));
        omega = AE_MUL(AE_MUL(2.0f, 3.14159265f), AE_SUB(1.0f, ctm));
        return;
    }
    const float4 h = ld4(b + 64);
    const f3 tl = P - from;
    const float d2 = fmax_(dot(tl, tl), 1e-8f);
    const float s = AE_ADD(AE_ADD(AE_MUL(h.x, h.y), AE_MUL(h.y, h.z)), AE_MUL(h.z, h.x));
    const float area = AE_DIV(AE_MUL(4.0f, s), 6.0f);
    omega = AE_DIV(area, d2);
}

// CalculateDirectLight, hybrid:1122-1212.
AE_DEV f3 direct_light(const DevScene &S, const DHit &h, f3 surf_albedo, float time, uint32_t &seed) {
    f3 acc = splat(0.0f);
    for (uint32_t i = 0; i < S.n_lights; i++) {
        const ae_object *L = S.objects + __ldg(S.lights + i);
        const ObjHead lh = load_head(L);
        f3 lp;
        float omega;
        sample_light(L, lh.shape, h.p, lp, omega, seed);
        if (omega <= 0.0f) continue;
        f3 sd = lp - h.p;
        const float dist = length(sd);
        if (dist <= 1e-6f) continue;
        sd = sd / dist;
        const float ct = dot(h.n, sd);
        if (ct <= 0.0f) continue;
        f3 so = h.p + h.n * 0.001f;
        bool occluded = false;
        for (int k = 0; k < 4; k++) {
            DHit sh;
            if (!traverse_ref(S, so, sd, time, 0.001f, sh, seed)) break;
            if (sh.t >= AE_SUB(distance(lp, so), 0.001f)) break;
            const uint32_t mt = load_head(S.objects + sh.slot).material;
            if (mt == AE_MAT_DIFFUSE_LIGHT) break;
            if (mt != AE_MAT_DIELECTRIC) { occluded = true; break; }
            so = sh.p + sd * 0.001f;
        }
        if (!occluded) {
            const MatRec lm = load_mat(L);
            const f3 rad = lm.emission * lm.albedo;
            acc = acc + surf_albedo * rad * ct * omega;
        }
    }
    return acc;
}

// GetBounce, hybrid:965-1033.
AE_DEV bool get_bounce(f3 d, const DHit &h, const MatRec &m, f3 &dir, uint32_t &seed) {
    dir = splat(0.0f);
    switch (m.type) {
    case AE_MAT_LAMBERTIAN:
        dir = h.n + random_direction(seed);
        if (dot(dir, dir) < 0.001f) dir = h.n;
        return true;
    case AE_MAT_METAL:
        dir = normalize(reflect(d, h.n));
        dir = dir + random_direction(seed) * m.fuzz;
        return dot(dir, h.n) > 0.0f;
    case AE_MAT_DIELECTRIC: {
        const float ri = h.front ? AE_DIV(1.0f, m.refraction) : m.refraction;
        const f3 dn = normalize(d);
        const float ct = fmin_(dot(-dn, h.n), 1.0f);
        const float st = AE_SQRT(fmax_(0.0f, AE_SUB(1.0f, AE_MUL(ct, ct))));
        const float r0 = powf_(AE_DIV(AE_SUB(1.0f, ri), AE_ADD(1.0f, ri)), 2.0f);
        const float refl = AE_ADD(r0, AE_MUL(AE_SUB(1.0f, r0), powf_(AE_SUB(1.0f, ct), 5.0f)));
        if (AE_MUL(ri, st) > 1.0f || refl > rng_next(seed)) dir = reflect(dn, h.n);
        else dir = refract(dn, h.n, ri);
        return true;
    }
    case AE_MAT_ISOTROPIC:
        dir = random_direction(seed);
        return true;
    default:
        return false;
    }
}

// ColorRay, hybrid:1230-1325.
AE_DEV f3 color_ray(const DevScene &S, const FrameParams &F, f3 o, f3 d, float time, uint32_t &seed) {
    f3 thr = splat(1.0f), acc = splat(0.0f);
    for (uint32_t b = 0; b < F.depth; b++) {
        DHit h;
        if (!traverse_ref(S, o, d, time, 0.001f, h, seed)) {
            acc = acc + thr * F.sky;
            break;
        }
        const MatRec m = load_mat(S.objects + h.slot);
        if (m.type == AE_MAT_DIFFUSE_LIGHT) {
            acc = acc + thr * (m.emission * m.albedo);
            break;
        }
        if (m.type == AE_MAT_LAMBERTIAN) {
            f3 dl = direct_light(S, h, m.albedo, time, seed);
            const float luma = maxc(dl);
            if (luma > 8.0f) dl = dl * AE_DIV(8.0f, luma);
            acc = acc + thr * dl;
        }
        f3 sd;
        if (!get_bounce(d, h, m, sd, seed)) break;
        d = normalize(sd);
        const float sgn = dot(d, h.n) < 0.0f ? -1.0f : 1.0f;
        o = h.p + h.n * AE_MUL(0.001f, sgn);
        if (m.type != AE_MAT_DIELECTRIC) thr = thr * m.albedo;
        if (b > 0) {
            const float p = clampf(maxc(thr), 0.1f, 1.0f);
            if (rng_next(seed) > p) break;
            thr = thr / p;
        }
    }
    return acc;
}

// ToneMapACES + LinearToSRGB (hybrid:213-233) into 8-bit sRGB.
AE_DEV uchar4 display_texel(f3 lin, float exposure) {
    const f3 x = lin * exposure;
    const f3 num = x * (2.51f * x + 0.03f);
    const f3 den = x * (2.43f * x + 0.59f) + 0.14f;
    f3 c = saturate(num / den);
    c = saturate(c);
    float out[3] = {c.x, c.y, c.z};
    unsigned char q[3];
    for (int k = 0; k < 3; k++) {
        const float v = out[k];
        const float s = v <= 0.0031308f ? AE_MUL(v, 12.92f)
                                        : AE_SUB(AE_MUL(1.055f, powf_(v, AE_DIV(1.0f, 2.4f))), 0.055f);
        q[k] = (unsigned char)(int)AE_RINT(AE_MUL(saturate(s), 255.0f));
    }
    return make_uchar4(q[0], q[1], q[2], 255);
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

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------
cudaError_t launch_closest_plain(const DevScene &S, const ae_ray *rays, uint32_t n, ae_hit *hits, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    k_closest_plain<<<(n + 127) / 128, 128, 0, st>>>(S, rays, n, hits);
    return cudaGetLastError();
}

cudaError_t launch_count_plain(const DevScene &S, const ae_ray *rays, uint32_t n, unsigned long long *totals,
                               cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    k_count_plain<<<(n + 127) / 128, 128, 0, st>>>(S, rays, n, totals);
    return cudaGetLastError();
}

cudaError_t launch_render_plain(const DevScene &S, const FrameParams &F, float4 *accum, uchar4 *display, float4 *frame,
                                cudaStream_t st) {
    dim3 grid((F.width + 15) / 16, (F.height + 7) / 8);
    k_render_plain<<<grid, 128, 0, st>>>(S, F, accum, display, frame);
    return cudaGetLastError();
}

}  // namespace ae
