// wf_common.cuh - device pieces shared by the queue-driven path tracers (the
// wavefront frame renderer and the serving loop): warp-aggregated queue
// appends, bulk-copy staging on an mbarrier, and ColorRay's per-vertex work
// (hybrid:1230-1325) split at the traversals so the shadow tests can run as
// their own queue.
//
// Every arithmetic step is the plain megakernel's (trace_plain.cu,
// color_ray), in the same order, so a path traced through these pieces gives
// the plain kernel's radiance bit for bit.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "bulk.cuh"
#include "fast_trace.cuh"
#include "shade.cuh"
#include "trace_common.cuh"

namespace ae {

// ---------------------------------------------------------------------------
// Warp-aggregated queue append: one atomic per warp, lanes get consecutive
// slots in lane order.
// ---------------------------------------------------------------------------
AE_DEV uint32_t warp_append(uint32_t *counter, uint32_t want) {
    const uint32_t lane = threadIdx.x & 31;
    const unsigned mask = __activemask();
    // inclusive prefix of `want` over the active lanes
    uint32_t incl = want;
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t v = __shfl_up_sync(mask, incl, off);
        if (lane >= uint32_t(off) && ((mask >> (lane - off)) & 1u)) incl += v;
    }
    const int leader = 31 - __clz(mask);  // highest active lane holds the total
    uint32_t base = 0;
    if (int(lane) == leader) base = atomicAdd(counter, incl);
    base = __shfl_sync(mask, base, leader);
    return base + incl - want;
}

// ---------------------------------------------------------------------------
// ColorRay split at its traversals
// ---------------------------------------------------------------------------

// Light samples of one path vertex: entry e holds the shadow ray (origin +
// tnear, direction + time), the sampled light point, the contribution if
// unoccluded, and the valid / occluded flags.
struct ShadowStore {
    float4 *o, *d, *lp, *c;
    uint8_t *valid, *occ;
};

// The precision form's shading data: per triangle record (in the optimised
// BVH's slot order) the three vertex normals and UVs as FP16, 32 bytes:
//   word 0: n0.x n0.y | n0.z n1.x | n1.y n1.z | n2.x n2.y
//   word 1: n2.z u0   | v0   u1   | v1   u2   | v2   (pad)
struct PrecView {
    const uint4 *shade16;  // 2 per triangle
};

AE_DEV float half_lo(uint32_t w) { return __half2float(__ushort_as_half((unsigned short)(w & 0xffffu))); }
AE_DEV float half_hi(uint32_t w) { return __half2float(__ushort_as_half((unsigned short)(w >> 16))); }

// surface_from_hit for the precision form: mesh hits take the shading normal
// from the FP16 record and the geometric normal from the optimised
// triangle record (the same FP32 positions); everything else as the plain form.
AE_DEV bool surface_from_hit_prec(const DevScene &S, const FastView &V, const PrecView &P, const ae_hit &h, f3 o,
                                  f3 d, float time, DHit &out) {
    if (h.object == AE_MISS) return false;
    const uint4 m = __ldg(V.meta + h.object);
    if ((m.x & 0xffu) != AE_SHAPE_MESH) return surface_from_hit(S, h, o, d, time, out);
    out.t = h.t;
    out.slot = h.object;
    out.prim = h.prim;
    out.alpha = h.alpha;
    out.beta = h.beta;
    out.p = o + d * h.t;
    const float4 *ip = reinterpret_cast<const float4 *>(V.inst + m.y);
    const float4 q = __ldg(ip + 1), rb = __ldg(ip + 2);
    const size_t tri = size_t(__float_as_uint(rb.y)) + h.prim;
    const float4 *tp = V.tris + 3 * tri;
    const float4 t0 = __ldg(tp), t1 = __ldg(tp + 1), t2 = __ldg(tp + 2);
    const f3 p0 = mk(t0.x, t0.y, t0.z), p1 = mk(t0.w, t1.x, t1.y), p2 = mk(t1.z, t1.w, t2.x);
    const uint4 s0 = __ldg(P.shade16 + 2 * tri), s1 = __ldg(P.shade16 + 2 * tri + 1);
    const f3 n0 = mk(half_lo(s0.x), half_hi(s0.x), half_lo(s0.y));
    const f3 n1 = mk(half_hi(s0.y), half_lo(s0.z), half_hi(s0.z));
    const f3 n2 = mk(half_lo(s0.w), half_hi(s0.w), half_lo(s1.x));
    const float w0 = AE_SUB(AE_SUB(1.0f, h.alpha), h.beta);
    const f3 sh = normalize(w0 * n0 + h.alpha * n1 + h.beta * n2);
    const f3 gn = cross(p1 - p0, p2 - p0);
    f3 geo = gn / AE_SQRT(dot(gn, gn));
    if (dot(geo, sh) < 0.0f) geo = -geo;
    out.front = dot(d, quat_rotate(q.x, q.y, q.z, q.w, geo)) < 0.0f;
    out.n = normalize(quat_rotate(q.x, q.y, q.z, q.w, sh));
    if (!out.front) out.n = -out.n;
    return true;
}

// Everything at one path vertex after its closest hit: sky or emission on a
// miss or a light, the light samples of a Lambertian surface (entries
// e0 .. e0 + n_lights - 1, throughput at the vertex into *pend, *nee set),
// then the bounce and Russian roulette.  Returns whether the path goes on,
// with its next ray in `nr`; `n_shadow` counts the valid light samples.
// PREC selects the precision form's FP16 shading normals.
template <bool PREC>
AE_DEV bool shade_vertex(const DevScene &S, const FastView &V, const PrecView &PV, const f3 &sky, uint32_t depth,
                         uint32_t n_lights, int bounce, const ae_ray &r, const ae_hit &hr, f3 &thr, f3 &acc,
                         uint32_t &seed, const ShadowStore &SH, size_t e0, uint8_t *nee, float4 *pend,
                         uint32_t &n_shadow, ae_ray &nr) {
    const f3 o = mk(r.ox, r.oy, r.oz), d = mk(r.dx, r.dy, r.dz);
    n_shadow = 0;
    nr = r;
    DHit h;
    const bool hit = PREC ? surface_from_hit_prec(S, V, PV, hr, o, d, r.time, h) : surface_from_hit(S, hr, o, d, r.time, h);
    if (!hit) {
        acc = acc + thr * sky;
        return false;
    }
    const MatRec m = load_mat(S.objects + h.slot);
    if (m.type == AE_MAT_DIFFUSE_LIGHT) {
        acc = acc + thr * (m.emission * m.albedo);
        return false;
    }
    // SurfaceAlbedo (textured when the material has a layer).
    const f3 alb = m.type != AE_MAT_DIELECTRIC ? surface_albedo(S, h, m, o, d) : m.albedo;
    if (m.type == AE_MAT_LAMBERTIAN) {
        // Light samples in light order (CalculateDirectLight,
        // hybrid:1122-1212); occlusion is resolved by the shadow stage.
        *nee = 1;
        *pend = make_float4(thr.x, thr.y, thr.z, 0.0f);
        for (uint32_t i = 0; i < n_lights; i++) {
            const size_t e = e0 + i;
            const ae_object *L = S.objects + __ldg(S.lights + i);
            const ObjHead lh = load_head(L);
            f3 lp;
            float omega;
            sample_light(L, lh.shape, h.p, lp, omega, seed);
            uint8_t valid = 0;
            if (omega > 0.0f) {
                f3 sd = lp - h.p;
                const float dist = length(sd);
                if (dist > 1e-6f) {
                    sd = sd / dist;
                    const float ct = dot(h.n, sd);
                    if (ct > 0.0f) {
                        const MatRec lm = load_mat(L);
                        const f3 rad = lm.emission * lm.albedo;
                        const f3 c = alb * rad * ct * omega;
                        const f3 so = h.p + h.n * 0.001f;
                        SH.o[e] = make_float4(so.x, so.y, so.z, 0.001f);
                        SH.d[e] = make_float4(sd.x, sd.y, sd.z, r.time);
                        SH.lp[e] = make_float4(lp.x, lp.y, lp.z, 0.0f);
                        SH.c[e] = make_float4(c.x, c.y, c.z, 0.0f);
                        valid = 1;
                        n_shadow++;
                    }
                }
            }
            SH.valid[e] = valid;
            SH.occ[e] = 0;
        }
    }
    f3 sd, gw;
    if (!get_bounce(d, h, m, alb, sd, gw, seed)) return false;
    const f3 nd = normalize(sd);
    const float sgn = dot(nd, h.n) < 0.0f ? -1.0f : 1.0f;
    const f3 no = h.p + h.n * AE_MUL(0.001f, sgn);
    if (m.type == AE_MAT_GGX_METAL) thr = thr * gw;
    else if (m.type != AE_MAT_DIELECTRIC) thr = thr * alb;
    if (bounce > 0) {
        const float p = clampf(maxc(thr), 0.1f, 1.0f);
        if (rng_next(seed) > p) return false;
        thr = thr / p;
    }
    if (uint32_t(bounce + 1) >= depth) return false;
    nr.ox = no.x; nr.oy = no.y; nr.oz = no.z; nr.tnear = 0.001f;
    nr.dx = nd.x; nr.dy = nd.y; nr.dz = nd.z;
    return true;
}

// Writes the indices of the valid light samples e0 .. e0 + n_lights - 1 to
// the shadow queue from `base` on, in light order.
AE_DEV void push_shadow_entries(const ShadowStore &SH, uint32_t e0, uint32_t n_lights, uint32_t *sq, uint32_t base) {
    uint32_t j = 0;
    for (uint32_t i = 0; i < n_lights; i++)
        if (SH.valid[e0 + i]) sq[base + j++] = e0 + i;
}

// The reference's shadow test (hybrid:1167-1191): up to four closest hits,
// stepping through glass; lights and anything beyond the light point do not
// block.  WT selects the watertight triangle test.
template <bool WT = false>
AE_DEV bool shadow_occluded(const DevScene &S, const FastView &V, f3 so, const f3 &sd, const f3 &lp, float time,
                            uint2 *stk, int tid, int nthreads) {
    for (int step = 0; step < 4; step++) {
        const Best b = closest_fast<WT>(S, V, so, sd, 0.001f, time, stk, tid, nthreads);
        if (b.object == AE_MISS) return false;
        if (b.t >= AE_SUB(distance(lp, so), 0.001f)) return false;
        const uint32_t mt = load_head(S.objects + b.object).material;
        if (mt == AE_MAT_DIFFUSE_LIGHT) return false;
        if (mt != AE_MAT_DIELECTRIC) return true;
        so = (so + sd * b.t) + sd * 0.001f;
    }
    return false;
}

// NEE of one vertex: unoccluded contributions in light order, then the luma
// clamp of 8 (hybrid:1207-1210).
AE_DEV f3 nee_total(const ShadowStore &SH, size_t e0, uint32_t n_lights) {
    f3 dl = splat(0.0f);
    for (uint32_t i = 0; i < n_lights; i++) {
        const size_t e = e0 + i;
        if (SH.valid[e] && !SH.occ[e]) {
            const float4 c = SH.c[e];
            dl = dl + mk(c.x, c.y, c.z);
        }
    }
    const float luma = maxc(dl);
    if (luma > 8.0f) dl = dl * AE_DIV(8.0f, luma);
    return dl;
}

}  // namespace ae
