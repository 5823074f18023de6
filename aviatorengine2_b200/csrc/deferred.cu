// deferred.cu - the hybrid renderer's compute passes without a raster stack:
//
//   k_gbuffer   writes the G-buffer planes the raster pass would
//               (gbuffer.vert/frag.hlsl; targets renderer/renderer.cpp:370-421)
//               by ray casting the primary hit over what the rasterizer draws
//               (mesh instances and unrotated untextured solid boxes,
//               IsRasterProxy renderer/renderer.h:317-323).
//   k_deferred  the deferred resolve, deferred.comp.hlsl:1879-2010: primary
//               from the G-buffer plus a bounded analytic trace, NEE with
//               any-hit shadow rays, Depth-1 indirect bounces, then either
//               reprojected accumulation (full resolution) or demodulated
//               lighting into the reduced grid.
//   k_upsample  upsample.comp.hlsl:280-390: 2x2 bilateral gather from the
//               reduced grid, re-modulation, reprojection, tone map.
//
// Traversal follows deferred.comp's own rules, which differ from the
// compute-only shader's: closest hit visits the nearer child first
// (deferred:1027-1099, 733-750), shadows use an any-hit walk that ignores glass
// and lights (deferred:1115-1171, 812-854).  All arithmetic goes through
// ae_math.h, so results are bit-identical to the oracle's.
#include <cuda_runtime.h>

#include <cstring>

#include "context.h"
#include "fast.h"
#include "kernels.h"
#include "shade.cuh"
#include "trace_common.cuh"

namespace ae {

struct Deferred {
    DevBuf<float4> gpos, gnrm;     // RGBA32F position (w = object slot), normal (w = coverage)
    DevBuf<uchar4> galb;           // RGBA8 albedo (a = 0 view-dependent)
    DevBuf<float> gdepth;          // D32F depth
    DevBuf<float4> accum[2], geom[2];
    DevBuf<float4> reduced;
    uint32_t history = 0;          // slot written most recently (historyIndex)
    uint32_t red_w = 1, red_h = 1;
    bool have_gbuffer = false;
    bool last_deferred = false;
};

void destroy_deferred(Ctx *c) {
    delete c->deferred;
    c->deferred = nullptr;
}

struct DefParams {
    FrameParams F;
    float jitter_x, jitter_y, trace_scale, history_cap, fov, znear, zfar;
    uint32_t frame_index, history_reset, camera_moved, debug_view, reduced, ext_w, ext_h, spp;
    float prev_vp[16];
};

// ---------------------------------------------------------------------------
// Traversal of deferred.comp
// ---------------------------------------------------------------------------

// AABBEntry, deferred:635-646.
AE_DEV float aabb_entry(f3 o, f3 inv, f3 lo, f3 hi, float tn, float tf) {
    const f3 t0 = (lo - o) * inv, t1 = (hi - o) * inv;
    const f3 a = vmin(t0, t1), b = vmax(t0, t1);
    const float tmin = fmax_(fmax_(a.x, a.y), fmax_(a.z, tn));
    const float tmax = fmin_(fmin_(b.x, b.y), fmin_(b.z, tf));
    return tmin <= tmax ? tmin : 1e30f;
}

// HitMesh with nearest-first children, deferred:684-806.
AE_DEV bool hit_mesh_ordered(const DevScene &S, uint32_t ii, f3 o, f3 d, float tn, float tf, DHit &h) {
    const float4 *ip = reinterpret_cast<const float4 *>(S.instances + ii);
    const float4 i0 = __ldg(ip), i1 = __ldg(ip + 1), i2 = __ldg(ip + 2);
    const uint32_t vbase = __float_as_uint(i2.x), ibase = __float_as_uint(i2.y), bbase = __float_as_uint(i2.w);
    f3 lo = quat_rotate(-i1.x, -i1.y, -i1.z, i1.w, o - mk(i0.x, i0.y, i0.z));
    f3 ld = quat_rotate(-i1.x, -i1.y, -i1.z, i1.w, d);
    if (i0.w != 0.0f && i0.w != 1.0f) {
        const float inv = AE_DIV(1.0f, i0.w);
        lo = lo * inv;
        ld = ld * inv;
    }
    const f3 invd = 1.0f / ld;
    int stack[kBlasStack];
    int sp = 0;
    stack[sp++] = 0;
    bool found = false;
    float closest = tf, ba = 0.0f, bb = 0.0f;
    uint32_t best = 0;
    f3 bgeo = mk(0.0f, 0.0f, 1.0f);
    while (sp > 0) {
        const NodeBox n = load_node(S.blas, bbase + uint32_t(stack[--sp]));
        if (!slab_ref(lo, invd, n.lo, n.hi, tn, closest)) continue;
        if (n.count > 0) {
            for (int i = 0; i < n.count; ++i) {
                const uint32_t base = ibase + uint32_t(n.left + i) * 3u;
                const f3 p0 = vtx_pos(S.vertices, vbase + __ldg(S.indices + base));
                const f3 p1 = vtx_pos(S.vertices, vbase + __ldg(S.indices + base + 1));
                const f3 p2 = vtx_pos(S.vertices, vbase + __ldg(S.indices + base + 2));
                float t, a, b;
                f3 g;
                if (tri_ref(lo, ld, tn, closest, p0, p1, p2, t, a, b, g)) {
                    closest = t; found = true; ba = a; bb = b; best = base; bgeo = g;
                }
            }
        } else {
            const NodeBox L = load_node(S.blas, bbase + uint32_t(n.left)), R = load_node(S.blas, bbase + uint32_t(n.right));
            const float tl = aabb_entry(lo, invd, L.lo, L.hi, tn, closest);
            const float tr = aabb_entry(lo, invd, R.lo, R.hi, tn, closest);
            const bool lf = tl <= tr;
            if (fmax_(tl, tr) < 1e30f && sp < kBlasStack) stack[sp++] = lf ? n.right : n.left;
            if (fmin_(tl, tr) < 1e30f && sp < kBlasStack) stack[sp++] = lf ? n.left : n.right;
        }
    }
    if (!found) return false;
    const ae_vertex *A = S.vertices + vbase + __ldg(S.indices + best);
    const ae_vertex *B = S.vertices + vbase + __ldg(S.indices + best + 1);
    const ae_vertex *C = S.vertices + vbase + __ldg(S.indices + best + 2);
    const float4 a0 = ld4(A), b0 = ld4(B), c0 = ld4(C);
    const float4 a1 = ld4(reinterpret_cast<const char *>(A) + 16), b1 = ld4(reinterpret_cast<const char *>(B) + 16),
                 c1 = ld4(reinterpret_cast<const char *>(C) + 16);
    const float w0 = AE_SUB(AE_SUB(1.0f, ba), bb);
    const f3 sh = normalize(w0 * mk(a0.w, a1.x, a1.y) + ba * mk(b0.w, b1.x, b1.y) + bb * mk(c0.w, c1.x, c1.y));
    f3 geo = bgeo;
    if (dot(geo, sh) < 0.0f) geo = -geo;
    h.t = closest;
    h.p = o + d * closest;
    h.n = normalize(quat_rotate(i1.x, i1.y, i1.z, i1.w, sh));
    h.front = dot(d, quat_rotate(i1.x, i1.y, i1.z, i1.w, geo)) < 0.0f;
    if (!h.front) h.n = -h.n;
    h.prim = (best - ibase) / 3u;
    h.alpha = ba;
    h.beta = bb;
    return true;
}

// OccludedMesh, deferred:812-854.
AE_DEV bool occluded_mesh(const DevScene &S, uint32_t ii, f3 o, f3 d, float tn, float tf) {
    const float4 *ip = reinterpret_cast<const float4 *>(S.instances + ii);
    const float4 i0 = __ldg(ip), i1 = __ldg(ip + 1), i2 = __ldg(ip + 2);
    const uint32_t vbase = __float_as_uint(i2.x), ibase = __float_as_uint(i2.y), bbase = __float_as_uint(i2.w);
    f3 lo = quat_rotate(-i1.x, -i1.y, -i1.z, i1.w, o - mk(i0.x, i0.y, i0.z));
    f3 ld = quat_rotate(-i1.x, -i1.y, -i1.z, i1.w, d);
    if (i0.w != 0.0f && i0.w != 1.0f) {
        const float inv = AE_DIV(1.0f, i0.w);
        lo = lo * inv;
        ld = ld * inv;
    }
    const f3 invd = 1.0f / ld;
    int stack[kBlasStack];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
        const NodeBox n = load_node(S.blas, bbase + uint32_t(stack[--sp]));
        if (!slab_ref(lo, invd, n.lo, n.hi, tn, tf)) continue;
        if (n.count > 0) {
            for (int i = 0; i < n.count; ++i) {
                const uint32_t base = ibase + uint32_t(n.left + i) * 3u;
                const f3 p0 = vtx_pos(S.vertices, vbase + __ldg(S.indices + base));
                const f3 p1 = vtx_pos(S.vertices, vbase + __ldg(S.indices + base + 1));
                const f3 p2 = vtx_pos(S.vertices, vbase + __ldg(S.indices + base + 2));
                float t, a, b;
                f3 g;
                if (tri_ref(lo, ld, tn, tf, p0, p1, p2, t, a, b, g)) return true;
            }
        } else if (sp + 2 <= kBlasStack) {
            stack[sp++] = n.left;
            stack[sp++] = n.right;
        }
    }
    return false;
}

// IsRasterProxy, deferred:1011-1017 (renderer/renderer.h:317-323).
AE_DEV bool is_raster_proxy(const ae_object *obj, const ObjHead &hd) {
    return hd.shape == AE_SHAPE_BOX && hd.material != AE_MAT_ISOTROPIC && hd.texture == AE_NO_TEXTURE &&
           ld4(reinterpret_cast<const char *>(obj) + 64).w == 0.0f;
}

AE_DEV bool hit_object_deferred(const DevScene &S, const ae_object *obj, const ObjHead &hd, f3 o, f3 d, float time,
                                float tn, float tf, DHit &h, uint32_t &seed) {
    if (hd.material == AE_MAT_ISOTROPIC) return hit_volume_ref(obj, hd.shape, o, d, time, tn, tf, h, seed);
    if (hd.shape == AE_SHAPE_SPHERE) return hit_sphere_ref(obj, o, d, time, tn, tf, h);
    if (hd.shape == AE_SHAPE_QUAD) return hit_planar_ref(obj, false, o, d, tn, tf, h);
    if (hd.shape == AE_SHAPE_TRIANGLE) return hit_planar_ref(obj, true, o, d, tn, tf, h);
    if (hd.shape == AE_SHAPE_MESH) {
        const uint32_t ii = __float_as_uint(ld4(reinterpret_cast<const char *>(obj) + 80).z);
        return hit_mesh_ordered(S, ii, o, d, tn, tf, h);
    }
    return hit_box_ref(obj, o, d, tn, tf, h);
}

// TraverseBVHBounded, deferred:1027-1099.
AE_DEV bool traverse_bounded(const DevScene &S, f3 o, f3 d, float time, float tn, float far_limit, bool skip_raster,
                             DHit &out, uint32_t &seed) {
    if (S.n_nodes == 0) return false;
    const f3 inv = 1.0f / d;
    int stack[kTlasStack];
    int sp = 0;
    stack[sp++] = 0;
    bool found = false;
    float tf = far_limit;
    while (sp > 0) {
        const NodeBox n = load_node(S.tlas, uint32_t(stack[--sp]));
        if (!slab_ref(o, inv, n.lo, n.hi, tn, tf)) continue;
        if (n.count > 0) {
            for (int i = 0; i < n.count; i++) {
                const uint32_t slot = uint32_t(n.left + i);
                const ae_object *obj = S.objects + slot;
                const ObjHead hd = load_head(obj);
                if (skip_raster && (hd.shape == AE_SHAPE_MESH || is_raster_proxy(obj, hd))) continue;
                DHit h;
                if (hit_object_deferred(S, obj, hd, o, d, time, tn, tf, h, seed)) {
                    tf = h.t;
                    h.slot = slot;
                    out = h;
                    found = true;
                }
            }
        } else {
            const NodeBox L = load_node(S.tlas, uint32_t(n.left)), R = load_node(S.tlas, uint32_t(n.right));
            const float tl = aabb_entry(o, inv, L.lo, L.hi, tn, tf);
            const float tr = aabb_entry(o, inv, R.lo, R.hi, tn, tf);
            const bool lf = tl <= tr;
            if (fmax_(tl, tr) < 1e30f && sp < kTlasStack) stack[sp++] = lf ? n.right : n.left;
            if (fmin_(tl, tr) < 1e30f && sp < kTlasStack) stack[sp++] = lf ? n.left : n.right;
        }
    }
    return found;
}

// Occluded, deferred:1115-1171.
AE_DEV bool occluded(const DevScene &S, f3 o, f3 d, float time, float tn, float tf, uint32_t &seed) {
    if (S.n_nodes == 0) return false;
    const f3 inv = 1.0f / d;
    int stack[kTlasStack];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
        const NodeBox n = load_node(S.tlas, uint32_t(stack[--sp]));
        if (!slab_ref(o, inv, n.lo, n.hi, tn, tf)) continue;
        if (n.count > 0) {
            for (int i = 0; i < n.count; i++) {
                const uint32_t slot = uint32_t(n.left + i);
                const ae_object *obj = S.objects + slot;
                const ObjHead hd = load_head(obj);
                if (hd.material == AE_MAT_DIELECTRIC || hd.material == AE_MAT_DIFFUSE_LIGHT) continue;
                if (hd.shape == AE_SHAPE_MESH) {
                    const uint32_t ii = __float_as_uint(ld4(reinterpret_cast<const char *>(obj) + 80).z);
                    if (occluded_mesh(S, ii, o, d, tn, tf)) return true;
                    continue;
                }
                DHit h;
                if (hit_object_deferred(S, obj, hd, o, d, time, tn, tf, h, seed)) return true;
            }
        } else if (sp + 2 <= kTlasStack) {
            stack[sp++] = n.left;
            stack[sp++] = n.right;
        }
    }
    return false;
}

// ---------------------------------------------------------------------------
// Shading of deferred.comp
// ---------------------------------------------------------------------------
struct SurfRec {  // the Hit of deferred.comp: geometry plus the material it shades with
    f3 p, n;
    bool front;
    uint32_t slot;
    f3 albedo;  // Object.Albedo (the G-buffer's albedo for raster surfaces)
    f3 surf;    // SurfaceAlbedo (deferred:1194-1203): textured when the material has a layer
    float fuzz, emission, refraction;
    uint32_t type, shape;
};

AE_DEV SurfRec surf_from_hit(const DevScene &S, const DHit &h, f3 o, f3 d) {
    const char *b = reinterpret_cast<const char *>(S.objects + h.slot);
    const float4 m0 = ld4(b + 80), m1 = ld4(b + 96), m2 = ld4(b + 112);
    SurfRec s;
    s.p = h.p; s.n = h.n; s.front = h.front; s.slot = h.slot;
    s.albedo = mk(m1.x, m1.y, m1.z); s.fuzz = m1.w; s.emission = m0.y; s.refraction = m2.x;
    s.shape = __float_as_uint(m2.y); s.type = __float_as_uint(m2.z);
    s.surf = surface_albedo(S, h, load_mat(S.objects + h.slot), o, d);
    return s;
}

AE_DEV f3 rand_dir(uint32_t &seed) {
    const float z = AE_SUB(AE_MUL(rng_next(seed), 2.0f), 1.0f);
    const float a = AE_MUL(rng_next(seed), 6.2831853f);
    const float r = AE_SQRT(AE_SUB(1.0f, AE_MUL(z, z)));
    return mk(AE_MUL(r, cosf_(a)), AE_MUL(r, sinf_(a)), z);
}

// GetBounce, deferred:1219-1288 (identical to the compute-only rules).
AE_DEV bool bounce_dir(f3 d, const SurfRec &h, f3 &dir, uint32_t &seed) {
    dir = splat(0.0f);
    switch (h.type) {
    case AE_MAT_LAMBERTIAN:
        dir = h.n + rand_dir(seed);
        if (dot(dir, dir) < 0.001f) dir = h.n;
        return true;
    case AE_MAT_METAL:
        dir = normalize(reflect(d, h.n));
        dir = dir + rand_dir(seed) * h.fuzz;
        return dot(dir, h.n) > 0.0f;
    case AE_MAT_DIELECTRIC: {
        const float ri = h.front ? AE_DIV(1.0f, h.refraction) : h.refraction;
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
        dir = rand_dir(seed);
        return true;
    default:
        return false;
    }
}

// SampleLight, deferred:1311-1373.
AE_DEV void sample_light_d(const ae_object *L, uint32_t shape, f3 from, f3 &p, float &omega, uint32_t &seed) {
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
        omega = AE_DIV(AE_MUL(AE_FABS(dot(ln, ts)), area), fmax_(d2, 1e-8f));
        return;
    }
    if (shape == AE_SHAPE_SPHERE) {
        const float radius = ld4(b + 16).w;
        const f3 tl = P - from;
        const float d2 = fmax_(dot(tl, tl), 1e-8f);
        const float r2 = AE_MUL(radius, radius);
        if (d2 <= r2) { omega = AE_MUL(4.0f, 3.14159265f); return; }
        omega = AE_MUL(AE_MUL(2.0f, 3.14159265f), AE_SUB(1.0f, AE_SQRT(fmax_(0.0f, AE_SUB(1.0f, AE_DIV(r2, d2))))));
        return;
    }
    const float4 h = ld4(b + 64);
    const f3 tl = P - from;
    const float d2 = fmax_(dot(tl, tl), 1e-8f);
    const float s = AE_ADD(AE_ADD(AE_MUL(h.x, h.y), AE_MUL(h.y, h.z)), AE_MUL(h.z, h.x));
    omega = AE_DIV(AE_DIV(AE_MUL(4.0f, s), 6.0f), d2);
}

// CalculateDirectLight with the any-hit shadow ray, deferred:1376-1446, then
// the clamp of ClampedDirectLight, deferred:1556-1569.
AE_DEV f3 clamped_direct(const DevScene &S, const SurfRec &h, float time, uint32_t &seed) {
    f3 acc = splat(0.0f);
    for (uint32_t i = 0; i < S.n_lights; i++) {
        const ae_object *L = S.objects + __ldg(S.lights + i);
        const ObjHead lh = load_head(L);
        f3 lp;
        float omega;
        sample_light_d(L, lh.shape, h.p, lp, omega, seed);
        if (omega <= 0.0f) continue;
        f3 sd = lp - h.p;
        const float dist = length(sd);
        if (dist <= 1e-6f) continue;
        sd = sd / dist;
        const float ct = dot(h.n, sd);
        if (ct <= 0.0f) continue;
        const f3 so = h.p + h.n * 0.001f;
        if (!occluded(S, so, sd, time, 0.001f, AE_SUB(dist, 0.001f), seed)) {
            const char *lb = reinterpret_cast<const char *>(L);
            const float4 m0 = ld4(lb + 80), m1 = ld4(lb + 96);
            const f3 rad = m0.y * mk(m1.x, m1.y, m1.z);
            acc = acc + h.surf * rad * ct * omega;
        }
    }
    const float luma = maxc(acc);
    if (luma > 8.0f) acc = acc * AE_DIV(8.0f, luma);
    return acc;
}

// TraceIndirect, deferred:1575-1646.
AE_DEV f3 trace_indirect(const DevScene &S, const DefParams &P, f3 pd, float time, const SurfRec &surf,
                         uint32_t &seed) {
    f3 bd;
    if (!bounce_dir(pd, surf, bd, seed)) return splat(0.0f);
    f3 d = normalize(bd);
    const float s0 = dot(d, surf.n) < 0.0f ? -1.0f : 1.0f;
    f3 o = surf.p + surf.n * AE_MUL(0.001f, s0);
    f3 thr = surf.type != AE_MAT_DIELECTRIC ? surf.surf : splat(1.0f);
    f3 acc = splat(0.0f);
    for (uint32_t b = 1; b < P.F.depth; b++) {
        DHit h;
        if (!traverse_bounded(S, o, d, time, 0.001f, 1000000.0f, false, h, seed)) {
            acc = acc + thr * P.F.sky;
            break;
        }
        const SurfRec s = surf_from_hit(S, h, o, d);
        if (s.type == AE_MAT_DIFFUSE_LIGHT) {
            acc = acc + thr * (s.emission * s.albedo);
            break;
        }
        if (s.type == AE_MAT_LAMBERTIAN) acc = acc + thr * clamped_direct(S, s, time, seed);
        f3 nx;
        if (!bounce_dir(d, s, nx, seed)) break;
        d = normalize(nx);
        const float sg = dot(d, s.n) < 0.0f ? -1.0f : 1.0f;
        o = s.p + s.n * AE_MUL(0.001f, sg);
        if (s.type != AE_MAT_DIELECTRIC) thr = thr * s.surf;
        const float p = clampf(maxc(thr), 0.1f, 1.0f);
        if (rng_next(seed) > p) break;
        thr = thr / p;
    }
    return acc;
}

// ---------------------------------------------------------------------------
// Reprojection shared by both passes (deferred:1759-1875, upsample:124-278)
// ---------------------------------------------------------------------------
struct Q4 {
    float x, y, z, w;
};
AE_DEV Q4 current_rotation(const DevScene &S, const ae_object *o) {
    const char *b = reinterpret_cast<const char *>(o);
    const float4 m2 = ld4(b + 112);
    const uint32_t shape = __float_as_uint(m2.y);
    if (shape == AE_SHAPE_MESH) {
        const uint32_t ii = __float_as_uint(ld4(b + 80).z);
        const float4 q = ld4(reinterpret_cast<const char *>(S.instances + ii) + 16);
        return Q4{q.x, q.y, q.z, q.w};
    }
    if (shape == AE_SHAPE_SPHERE || shape == AE_SHAPE_BOX) {
        const float half = AE_MUL(0.5f, ld4(b + 64).w);
        return Q4{0.0f, sinf_(half), 0.0f, cosf_(half)};
    }
    return Q4{0.0f, 0.0f, 0.0f, 1.0f};
}
AE_DEV f3 previous_position(const DevScene &S, const ae_object *o, f3 pos) {
    const char *b = reinterpret_cast<const char *>(o);
    const float4 q0 = ld4(b), q1 = ld4(b + 16), q2 = ld4(b + 32), q3 = ld4(b + 48);
    const Q4 r = current_rotation(S, o);
    const f3 local = quat_rotate(-r.x, -r.y, -r.z, r.w, pos - mk(q0.x, q0.y, q0.z));
    const f3 v = mk(q0.w, q2.w, q3.w);  // PrevRotX/Y/Z at offsets 12, 44, 60
    const float w = AE_SQRT(fmax_(0.0f, AE_SUB(1.0f, dot(v, v))));
    return quat_rotate(v.x, v.y, v.z, w, local) + mk(q1.x, q1.y, q1.z);
}

AE_DEV void reproject(const DefParams &P, uint32_t px, uint32_t py, f3 color, bool surface, f3 position, f3 prev_pos,
                      f3 normal, bool view_dep, const float4 *prev_img, const float4 *prev_geo, f3 &result,
                      float &count) {
    const uint32_t W = P.F.width, H = P.F.height;
    int hx = int(px), hy = int(py);
    bool valid = P.history_reset == 0;
    if (valid && P.camera_moved != 0) {
        valid = false;
        if (surface) {
            const float *m = P.prev_vp;
            const float v[4] = {prev_pos.x, prev_pos.y, prev_pos.z, 1.0f};
            float clip[4];
            for (int r = 0; r < 4; r++)
                clip[r] = AE_ADD(AE_ADD(AE_ADD(AE_MUL(m[4 * r], v[0]), AE_MUL(m[4 * r + 1], v[1])),
                                        AE_MUL(m[4 * r + 2], v[2])), AE_MUL(m[4 * r + 3], v[3]));
            if (clip[3] > 0.0f) {
                const float ux = AE_ADD(AE_MUL(AE_DIV(clip[0], clip[3]), 0.5f), 0.5f);
                const float uy = AE_ADD(AE_MUL(AE_DIV(clip[1], clip[3]), -0.5f), 0.5f);
                const float fx = AE_FLOOR(AE_MUL(ux, AE_U2F(W))), fy = AE_FLOOR(AE_MUL(uy, AE_U2F(H)));
                // int2(floor(...)): out-of-range values are rejected below
                // before any load; clamp the conversion itself to int range.
                hx = int(fmax_(fmin_(fx, 2.0e9f), -2.0e9f));
                hy = int(fmax_(fmin_(fy, 2.0e9f), -2.0e9f));
                if (hx >= 0 && hy >= 0 && hx < int(W) && hy < int(H)) {
                    const float4 prev = prev_geo[size_t(hy) * W + hx];
                    const f3 pp = mk(prev.x, prev.y, prev.z);
                    const float plane = AE_FABS(dot(pp - prev_pos, normal));
                    const float dist = length(position - P.F.source);
                    const float tol = AE_ADD(AE_MUL(0.01f, dist), 0.01f);
                    const float footprint =
                        AE_DIV(AE_MUL(AE_MUL(dist, 2.0f), tanf_(radians(AE_MUL(P.fov, 0.5f)))), AE_U2F(H));
                    const float facing = fmax_(AE_FABS(dot(normal, normalize(P.F.source - position))), 0.33f);
                    const float drift = length(pp - prev_pos);
                    valid = prev.w > 0.0f && plane < tol && drift < fmax_(AE_DIV(AE_MUL(2.5f, footprint), facing), 0.01f);
                }
            }
        }
    }
    if (!valid) {
        count = 1.0f;
        result = color;
        return;
    }
    const size_t hp = size_t(hy) * W + hx;
    const float prev_count = AE_FABS(prev_geo[hp].w);
    const float moving_cap = view_dep ? fmin_(P.history_cap, 4.0f) : P.history_cap;
    const float cap = P.camera_moved != 0 ? moving_cap : 1e7f;
    count = fmin_(AE_ADD(prev_count, 1.0f), cap);
    const float4 pi = prev_img[hp];
    result = lerp(mk(pi.x, pi.y, pi.z), color, AE_DIV(1.0f, count));
}

// ToneMapACES + LinearToSRGB into 8 bits (deferred:281-303).
AE_DEV uchar4 to_display(f3 lin, float exposure) {
    const f3 x = lin * exposure;
    f3 c = saturate((x * (2.51f * x + 0.03f)) / (x * (2.43f * x + 0.59f) + 0.14f));
    c = saturate(c);
    const float v[3] = {c.x, c.y, c.z};
    unsigned char q[3];
    for (int k = 0; k < 3; k++) {
        const float s = v[k] <= 0.0031308f ? AE_MUL(v[k], 12.92f)
                                           : AE_SUB(AE_MUL(1.055f, powf_(v[k], AE_DIV(1.0f, 2.4f))), 0.055f);
        q[k] = (unsigned char)(int)AE_RINT(AE_MUL(saturate(s), 255.0f));
    }
    return make_uchar4(q[0], q[1], q[2], 255);
}

// TracedTexel, deferred:1742-1747 and upsample:204-209.
AE_DEV void traced_texel(const DefParams &P, uint32_t cx, uint32_t cy, uint32_t &tx, uint32_t &ty) {
    const uint32_t k = P.frame_index % 4u;
    const float ox = (k == 1 || k == 2) ? 0.5f : 0.0f;
    const float oy = (k == 1 || k == 3) ? 0.5f : 0.0f;
    const float fx = AE_FLOOR(AE_DIV(AE_ADD(AE_U2F(cx), ox), P.trace_scale));
    const float fy = AE_FLOOR(AE_DIV(AE_ADD(AE_U2F(cy), oy), P.trace_scale));
    tx = min(uint32_t(fx), P.F.width - 1);
    ty = min(uint32_t(fy), P.F.height - 1);
}

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------
struct GBuf {
    float4 *pos, *nrm;
    uchar4 *alb;
    float *depth;
};
struct Images {
    float4 *img, *geo_out, *reduced;
    const float4 *prev_img, *prev_geo;
    uchar4 *display;
};

// The G-buffer through pixel centre + jitter: closest hit over the objects
// the rasterizer draws.  Writes zero coverage where nothing is drawn, as the
// raster pass clears its targets (renderer/renderer.cpp:1221-1233).
__global__ void __launch_bounds__(128) k_gbuffer(DevScene S, DefParams P, GBuf G) {
    const uint32_t x = blockIdx.x * 16 + (threadIdx.x & 15);
    const uint32_t y = blockIdx.y * 8 + (threadIdx.x >> 4);
    if (x >= P.F.width || y >= P.F.height) return;
    const size_t px = size_t(y) * P.F.width + x;
    const f3 sample = P.F.pixel0 + AE_ADD(AE_U2F(x), P.jitter_x) * P.F.pixel_u + AE_ADD(AE_U2F(y), P.jitter_y) * P.F.pixel_v;
    const f3 o = P.F.source, d = normalize(sample - o);
    // Closest hit over meshes and raster proxies: the reference's compute-only
    // walk restricted by shape.
    float4 pos = make_float4(0, 0, 0, 0), nrm = make_float4(0, 0, 0, 0);
    uchar4 alb = make_uchar4(0, 0, 0, 0);
    float depth = 1.0f;
    if (S.n_nodes > 0) {
        const f3 inv = 1.0f / d;
        int stack[kTlasStack];
        int sp = 0;
        stack[sp++] = 0;
        float tf = kFarStart;
        bool found = false;
        DHit best;
        while (sp > 0) {
            const NodeBox n = load_node(S.tlas, uint32_t(stack[--sp]));
            if (!slab_ref(o, inv, n.lo, n.hi, 0.001f, tf)) continue;
            if (n.count > 0) {
                for (int i = 0; i < n.count; i++) {
                    const uint32_t slot = uint32_t(n.left + i);
                    const ae_object *obj = S.objects + slot;
                    const ObjHead hd = load_head(obj);
                    DHit h;
                    bool hit = false;
                    if (hd.shape == AE_SHAPE_MESH) {
                        const uint32_t ii = __float_as_uint(ld4(reinterpret_cast<const char *>(obj) + 80).z);
                        hit = hit_mesh_ref(S, ii, o, d, 0.001f, tf, h);
                    } else if (is_raster_proxy(obj, hd)) {
                        hit = hit_box_ref(obj, o, d, 0.001f, tf, h);
                    }
                    if (hit) {
                        tf = h.t;
                        h.slot = slot;
                        best = h;
                        found = true;
                    }
                }
            } else if (sp + 2 <= kTlasStack) {
                stack[sp++] = n.left;
                stack[sp++] = n.right;
            }
        }
        if (found) {
            const ae_object *obj = S.objects + best.slot;
            const MatRec mat = load_mat(obj);
            const uint32_t type = mat.type;
            // SurfaceBlock's albedo (gbuffer.frag:44-50): textured at the
            // hit's UV when the material has a layer.
            const f3 sa = surface_albedo(S, best, mat, o, d);
            // The raster normal is the surface's own (outward), not flipped
            // toward the viewer: undo the intersector's facing flip.
            const f3 nn = best.front ? best.n : -best.n;
            pos = make_float4(best.p.x, best.p.y, best.p.z, AE_U2F(best.slot));
            nrm = make_float4(nn.x, nn.y, nn.z, 1.0f);
            const bool vd = type == AE_MAT_METAL || type == AE_MAT_DIELECTRIC;
            alb = make_uchar4((unsigned char)(int)AE_RINT(AE_MUL(saturate(sa.x), 255.0f)),
                              (unsigned char)(int)AE_RINT(AE_MUL(saturate(sa.y), 255.0f)),
                              (unsigned char)(int)AE_RINT(AE_MUL(saturate(sa.z), 255.0f)), vd ? 0 : 255);
            // PerspectiveRH_ZO depth (math/mat4.h:84-95) of the view-space z.
            const float vz = dot(best.p - o, -P.F.cam_w);
            depth = AE_DIV(AE_MUL(P.zfar, AE_SUB(P.znear, vz)), AE_MUL(AE_SUB(P.znear, P.zfar), vz));
        }
    }
    G.pos[px] = pos;
    G.nrm[px] = nrm;
    G.alb[px] = alb;
    G.depth[px] = depth;
}

// ResolvePrimary with HitFromGBuffer, deferred:1452-1548.  Returns 0 sky,
// 1 raster, 2 analytic.
AE_DEV int resolve_primary(const DevScene &S, const GBuf &G, size_t px, f3 o, f3 d, float time, SurfRec &hit,
                           uint32_t &seed) {
    SurfRec raster;
    bool has_raster = false;
    float far_limit = 1000000.0f;
    const float4 pn = G.nrm[px];
    if (!(pn.w < 0.5f)) {
        const float4 pp = G.pos[px];
        const uint32_t slot = uint32_t(AE_ADD(pp.w, 0.5f));
        if (slot < S.n_objects) {
            raster.p = mk(pp.x, pp.y, pp.z);
            raster.n = normalize(mk(pn.x, pn.y, pn.z));
            raster.slot = slot;
            const char *b = reinterpret_cast<const char *>(S.objects + slot);
            const float4 m0 = ld4(b + 80), m1 = ld4(b + 96), m2 = ld4(b + 112);
            const uchar4 a = G.alb[px];
            raster.albedo = mk(AE_DIV(AE_U2F(a.x), 255.0f), AE_DIV(AE_U2F(a.y), 255.0f), AE_DIV(AE_U2F(a.z), 255.0f));
            raster.surf = raster.albedo;  // HitFromGBuffer clears TextureID (deferred:1477-1480)
            raster.fuzz = m1.w; raster.emission = m0.y; raster.refraction = m2.x;
            raster.shape = __float_as_uint(m2.y); raster.type = __float_as_uint(m2.z);
            raster.front = dot(d, raster.n) < 0.0f;
            if (!raster.front) raster.n = -raster.n;
            far_limit = length(raster.p - o);
            has_raster = true;
        }
    }
    DHit ah;
    if (traverse_bounded(S, o, d, time, 0.001f, far_limit, true, ah, seed)) {
        hit = surf_from_hit(S, ah, o, d);
        return 2;
    }
    if (has_raster) {
        hit = raster;
        return 1;
    }
    return 0;
}

// MaterialFalseColour, deferred:1652-1663.
AE_DEV f3 false_colour(uint32_t t) {
    switch (t) {
    case AE_MAT_LAMBERTIAN: return mk(0.55f, 0.55f, 0.55f);
    case AE_MAT_METAL: return mk(1.0f, 0.75f, 0.1f);
    case AE_MAT_DIELECTRIC: return mk(0.1f, 0.85f, 1.0f);
    case AE_MAT_DIFFUSE_LIGHT: return mk(1.0f, 1.0f, 1.0f);
    case AE_MAT_ISOTROPIC: return mk(0.7f, 0.3f, 1.0f);
    default: return mk(1.0f, 0.0f, 1.0f);
    }
}

// DebugColour, deferred:1667-1722 (WorldFromDepth, deferred:1503-1514).
AE_DEV f3 debug_colour(const DevScene &S, const DefParams &P, const GBuf &G, size_t px, f3 o, f3 d, float time,
                       uint32_t &seed) {
    const float4 pn = G.nrm[px];
    const bool covered = pn.w >= 0.5f;
    const f3 background = mk(0.0f, 0.0f, 0.0f);
    if (P.debug_view == 1) {
        const uchar4 a = G.alb[px];
        return covered ? mk(AE_DIV(AE_U2F(a.x), 255.0f), AE_DIV(AE_U2F(a.y), 255.0f), AE_DIV(AE_U2F(a.z), 255.0f))
                       : background;
    }
    if (P.debug_view == 2) return covered ? mk(pn.x, pn.y, pn.z) * 0.5f + 0.5f : background;
    if (P.debug_view == 3) {
        if (!covered) return background;
        const float4 p = G.pos[px];
        return mk(fracf(AE_DIV(p.x, 100.0f)), fracf(AE_DIV(p.y, 100.0f)), fracf(AE_DIV(p.z, 100.0f)));
    }
    if (P.debug_view == 6) {
        if (!covered) return mk(0.0f, 0.0f, 0.2f);
        const float4 p = G.pos[px];
        const f3 stored = mk(p.x, p.y, p.z);
        const float dd = G.depth[px];
        const float vz = AE_DIV(AE_MUL(P.znear, P.zfar), AE_ADD(P.zfar, AE_MUL(dd, AE_SUB(P.znear, P.zfar))));
        const float t = AE_DIV(vz, dot(d, -P.F.cam_w));
        const f3 rebuilt = o + d * t;
        const float rel = AE_DIV(length(rebuilt - stored), fmax_(length(stored - o), 1e-4f));
        return splat(AE_MUL(rel, 100.0f));
    }
    SurfRec hit;
    const int source = resolve_primary(S, G, px, o, d, time, hit, seed);
    if (P.debug_view == 4) return source != 0 ? false_colour(hit.type) : background;
    if (source == 1) return mk(0.1f, 0.8f, 0.2f);
    if (source == 2) return mk(0.85f, 0.15f, 0.1f);
    return mk(0.1f, 0.15f, 0.5f);
}

__global__ void __launch_bounds__(128) k_deferred(DevScene S, DefParams P, GBuf G, Images I) {
    const uint32_t cx = blockIdx.x * 16 + (threadIdx.x & 15);
    const uint32_t cy = blockIdx.y * 8 + (threadIdx.x >> 4);
    if (cx >= P.ext_w || cy >= P.ext_h) return;
    uint32_t x = cx, y = cy;
    if (P.reduced) traced_texel(P, cx, cy, x, y);
    const size_t px = size_t(y) * P.F.width + x;
    if (P.F.display_only) {
        if (!P.reduced) {
            const float4 a = I.img[px];
            I.display[px] = to_display(mk(a.x, a.y, a.z), P.F.exposure);
        }
        return;
    }
    uint32_t seed = x + y * P.F.width + P.frame_index * P.F.width * P.F.height + 1u;
    const f3 sample = P.F.pixel0 + AE_ADD(AE_U2F(x), P.jitter_x) * P.F.pixel_u + AE_ADD(AE_U2F(y), P.jitter_y) * P.F.pixel_v;
    const f3 o = P.F.source;
    const f3 d = normalize(sample - o);
    const float time = rng_next(seed);
    if (P.debug_view != 0) {
        const f3 c = debug_colour(S, P, G, px, o, d, time, seed);
        const f3 q = saturate(c);
        I.display[px] = make_uchar4((unsigned char)(int)AE_RINT(AE_MUL(q.x, 255.0f)),
                                    (unsigned char)(int)AE_RINT(AE_MUL(q.y, 255.0f)),
                                    (unsigned char)(int)AE_RINT(AE_MUL(q.z, 255.0f)), 255);
        return;
    }
    // ResolvePrimary, deferred:1526-1548.
    f3 color = splat(0.0f);
    SurfRec hit;
    const int source = resolve_primary(S, G, px, o, d, time, hit, seed);
    const bool has = source != 0;
    if (!has) {
        color = P.F.sky;
    } else if (hit.type == AE_MAT_DIFFUSE_LIGHT) {
        color = hit.emission * hit.albedo;
    } else {
        for (uint32_t s = 0; s < P.spp; s++) {
            if (hit.type == AE_MAT_LAMBERTIAN) color = color + clamped_direct(S, hit, time, seed);
            color = color + trace_indirect(S, P, d, time, hit, seed);
        }
        color = color / AE_U2F(P.spp);
    }
    if (P.reduced) {
        const bool demod = source == 1 && hit.type != AE_MAT_DIELECTRIC;
        f3 alb = splat(1.0f);
        if (demod) alb = vmax(hit.surf, splat(0.01f));
        const f3 l = color / alb;
        I.reduced[size_t(cy) * P.ext_w + cx] = make_float4(l.x, l.y, l.z, demod ? 1.0f : 0.0f);
        return;
    }
    const bool surface = source != 0;
    const bool view_dep = surface && (hit.type == AE_MAT_METAL || hit.type == AE_MAT_DIELECTRIC);
    const f3 hp = has ? hit.p : mk(0.0f, 0.0f, 0.0f);
    const f3 prev = surface ? previous_position(S, S.objects + hit.slot, hit.p) : hp;
    f3 acc;
    float hl;
    reproject(P, x, y, color, surface, hp, prev, has ? hit.n : splat(0.0f), view_dep, I.prev_img, I.prev_geo, acc, hl);
    I.img[px] = make_float4(acc.x, acc.y, acc.z, 1.0f);
    I.geo_out[px] = make_float4(hp.x, hp.y, hp.z, surface ? hl : -hl);
    I.display[px] = to_display(acc, P.F.exposure);
}

__global__ void __launch_bounds__(128) k_upsample(DevScene S, DefParams P, GBuf G, Images I) {
    const uint32_t x = blockIdx.x * 16 + (threadIdx.x & 15);
    const uint32_t y = blockIdx.y * 8 + (threadIdx.x >> 4);
    if (x >= P.F.width || y >= P.F.height) return;
    const size_t px = size_t(y) * P.F.width + x;
    if (P.F.display_only) {
        const float4 a = I.img[px];
        I.display[px] = to_display(mk(a.x, a.y, a.z), P.F.exposure);
        return;
    }
    const int cmx = int(P.ext_w) - 1, cmy = int(P.ext_h) - 1;
    const float4 np = G.nrm[px];
    const bool cov_p = np.w > 0.5f;
    const float4 gp = G.pos[px];
    const float depth_p = length(mk(gp.x, gp.y, gp.z) - P.F.source);
    const uchar4 ap = G.alb[px];
    const f3 alb_p = mk(AE_DIV(AE_U2F(ap.x), 255.0f), AE_DIV(AE_U2F(ap.y), 255.0f), AE_DIV(AE_U2F(ap.z), 255.0f));
    const float cpx = AE_SUB(AE_MUL(AE_ADD(AE_U2F(x), 0.5f), P.trace_scale), 0.5f);
    const float cpy = AE_SUB(AE_MUL(AE_ADD(AE_U2F(y), 0.5f), P.trace_scale), 0.5f);
    const int bx = int(AE_FLOOR(cpx)), by = int(AE_FLOOR(cpy));
    f3 sum = splat(0.0f), nearest = splat(0.0f);
    float wsum = 0.0f, nd = 1e30f;
    for (int j = 0; j < 2; j++) {
        for (int i = 0; i < 2; i++) {
            const uint32_t cx = uint32_t(min(max(bx + i, 0), cmx)), cy = uint32_t(min(max(by + j, 0), cmy));
            uint32_t tx, ty;
            traced_texel(P, cx, cy, tx, ty);
            const size_t tp = size_t(ty) * P.F.width + tx;
            const float4 lit = I.reduced[size_t(cy) * P.ext_w + cx];
            const float4 nt = G.nrm[tp];
            const bool cov_t = nt.w > 0.5f;
            f3 alb = alb_p;
            if (!cov_p) {
                const uchar4 at = G.alb[tp];
                alb = mk(AE_DIV(AE_U2F(at.x), 255.0f), AE_DIV(AE_U2F(at.y), 255.0f), AE_DIV(AE_U2F(at.z), 255.0f));
            }
            const f3 rad = lit.w > 0.5f ? mk(lit.x, lit.y, lit.z) * alb : mk(lit.x, lit.y, lit.z);
            const float ox = AE_SUB(AE_U2F(tx), AE_U2F(x)), oy = AE_SUB(AE_U2F(ty), AE_U2F(y));
            const float d2 = AE_ADD(AE_MUL(ox, ox), AE_MUL(oy, oy));
            if (d2 < nd) { nd = d2; nearest = rad; }
            float w = expf_(AE_MUL(AE_MUL(-d2, P.trace_scale), P.trace_scale));
            if (cov_t != cov_p) {
                w = 0.0f;
            } else if (cov_p) {
                const float4 gt = G.pos[tp];
                const float depth_t = length(mk(gt.x, gt.y, gt.z) - P.F.source);
                w = AE_MUL(w, expf_(AE_DIV(-AE_FABS(AE_SUB(depth_p, depth_t)), AE_ADD(AE_MUL(0.01f, depth_p), 0.001f))));
                w = AE_MUL(w, powf_(saturate(dot(mk(np.x, np.y, np.z), mk(nt.x, nt.y, nt.z))), 32.0f));
            }
            sum = sum + w * rad;
            wsum = AE_ADD(wsum, w);
        }
    }
    const f3 color = wsum > 1e-4f ? sum / wsum : nearest;
    const f3 pos_p = mk(gp.x, gp.y, gp.z);
    const bool view_dep = cov_p && ap.w < 128;
    f3 prev = pos_p;
    if (cov_p) {
        const uint32_t slot = uint32_t(gp.w);
        if (slot < S.n_objects) prev = previous_position(S, S.objects + slot, pos_p);
    }
    f3 acc;
    float hl;
    reproject(P, x, y, color, cov_p, pos_p, prev, mk(np.x, np.y, np.z), view_dep, I.prev_img, I.prev_geo, acc, hl);
    I.img[px] = make_float4(acc.x, acc.y, acc.z, 1.0f);
    I.geo_out[px] = make_float4(pos_p.x, pos_p.y, pos_p.z, cov_p ? hl : -hl);
    I.display[px] = to_display(acc, P.F.exposure);
}

// ---------------------------------------------------------------------------
// Host
// ---------------------------------------------------------------------------
static uint32_t scaled_extent(uint32_t size, float scale) {
    // ScaledExtent, renderer/renderer.h:217-221
    return uint32_t(std::ceil(float(size) * scale));
}

static int ensure(Ctx *c) {
    if (!c->deferred) c->deferred = new (std::nothrow) Deferred();
    Deferred *D = c->deferred;
    if (!D) return c->fail(AE_ERR_OOM, "deferred state");
    const size_t px = size_t(c->settings.width) * c->settings.height;
    if (D->gpos.cap < px) {
        if (D->gpos.reserve(px) || D->gnrm.reserve(px) || D->galb.reserve(px) || D->gdepth.reserve(px) ||
            D->accum[0].reserve(px) || D->accum[1].reserve(px) || D->geom[0].reserve(px) || D->geom[1].reserve(px))
            return c->fail(AE_ERR_OOM, "deferred images");
        cudaMemsetAsync(D->gnrm.ptr, 0, px * sizeof(float4), c->stream);
        cudaMemsetAsync(D->gpos.ptr, 0, px * sizeof(float4), c->stream);
        cudaMemsetAsync(D->galb.ptr, 0, px * sizeof(uchar4), c->stream);
        for (int k = 0; k < 2; k++) {
            cudaMemsetAsync(D->accum[k].ptr, 0, px * sizeof(float4), c->stream);
            cudaMemsetAsync(D->geom[k].ptr, 0, px * sizeof(float4), c->stream);
        }
    }
    return AE_OK;
}

static DefParams make_def_params(const Ctx *c) {
    const ae_config &k = c->config;
    DefParams P;
    std::memset(&P, 0, sizeof(P));
    P.F = make_frame_params(k);
    P.F.depth = k.depth;
    P.jitter_x = k.jitter_x;
    P.jitter_y = k.jitter_y;
    P.trace_scale = k.traceScale > 0.0f ? k.traceScale : 1.0f;
    P.history_cap = k.historyCap;
    P.fov = k.fov;
    P.znear = k.zNear;
    P.zfar = k.zFar;
    P.frame_index = k.frameIndex;
    P.history_reset = k.historyReset;
    P.camera_moved = k.cameraMoved;
    P.debug_view = k.debugView;
    P.reduced = P.trace_scale < 1.0f ? 1u : 0u;
    P.ext_w = P.reduced ? scaled_extent(k.width, P.trace_scale) : k.width;
    P.ext_h = P.reduced ? scaled_extent(k.height, P.trace_scale) : k.height;
    const uint32_t per = k.batches ? k.samples / k.batches : k.samples;
    P.spp = per > 1u ? per : 1u;
    std::memcpy(P.prev_vp, k.prevViewProj, sizeof(P.prev_vp));
    return P;
}

int render_deferred(Ctx *c, const ae_gbuffer *gb) {
    int rc = ensure(c);
    if (rc) return rc;
    Deferred &D = *c->deferred;
    const DefParams P = make_def_params(c);
    const size_t px = size_t(c->settings.width) * c->settings.height;
    if (gb) {
        // Caller-provided G-buffer planes (the raster pass's output).
        const cudaMemcpyKind kind = gb->on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
        if (!gb->position || !gb->normal || !gb->albedo) return c->fail(AE_ERR_INVALID, "incomplete G-buffer");
        if ((rc = c->cuda(cudaMemcpyAsync(D.gpos.ptr, gb->position, px * 16, kind, c->stream), "G-buffer position")) ||
            (rc = c->cuda(cudaMemcpyAsync(D.gnrm.ptr, gb->normal, px * 16, kind, c->stream), "G-buffer normal")) ||
            (rc = c->cuda(cudaMemcpyAsync(D.galb.ptr, gb->albedo, px * 4, kind, c->stream), "G-buffer albedo")))
            return rc;
        if (gb->depth &&
            (rc = c->cuda(cudaMemcpyAsync(D.gdepth.ptr, gb->depth, px * 4, kind, c->stream), "G-buffer depth")))
            return rc;
        D.have_gbuffer = true;
    }
    if (!D.have_gbuffer) return c->fail(AE_ERR_STATE, "deferred resolve without a G-buffer (ae_build_gbuffer)");
    if (P.reduced) {
        const size_t rn = size_t(P.ext_w) * P.ext_h;
        if (D.reduced.reserve(rn)) return c->fail(AE_ERR_OOM, "reduced grid");
        D.red_w = P.ext_w;
        D.red_h = P.ext_h;
    }
    // renderer/renderer.cpp:1374-1378: history slots swap on frames that
    // write history (lit image, not converged).
    const bool writes = P.debug_view == 0 && !P.F.display_only;
    const uint32_t wslot = writes ? 1u - D.history : D.history;
    const uint32_t rslot = 1u - wslot;
    GBuf G{D.gpos.ptr, D.gnrm.ptr, D.galb.ptr, D.gdepth.ptr};
    Images I{D.accum[wslot].ptr, D.geom[wslot].ptr, D.reduced.ptr, D.accum[rslot].ptr, D.geom[rslot].ptr,
             c->display.ptr};
    if ((rc = c->timed_begin())) return rc;
    if (!(P.reduced && P.F.display_only)) {
        dim3 grid((P.ext_w + 15) / 16, (P.ext_h + 7) / 8);
        k_deferred<<<grid, 128, 0, c->stream>>>(c->scene(), P, G, I);
        if ((rc = c->cuda(cudaGetLastError(), "deferred launch"))) return rc;
        c->launches++;
    }
    if (P.reduced) {
        dim3 grid((P.F.width + 15) / 16, (P.F.height + 7) / 8);
        k_upsample<<<grid, 128, 0, c->stream>>>(c->scene(), P, G, I);
        if ((rc = c->cuda(cudaGetLastError(), "upsample launch"))) return rc;
        c->launches++;
    }
    c->launches--;  // timed_end counts one launch
    if ((rc = c->timed_end())) return rc;
    if (writes) D.history = wslot;
    D.last_deferred = true;
    return AE_OK;
}

int read_image_extra(Ctx *c, int which, void *dst, size_t bytes) {
    Deferred *D = c->deferred;
    const size_t px = size_t(c->settings.width) * c->settings.height;
    const void *src = nullptr;
    size_t need = 0;
    switch (which) {
    case AE_IMAGE_REDUCED:
        if (!D || !D->reduced.ptr) return c->fail(AE_ERR_STATE, "no reduced grid yet");
        src = D->reduced.ptr;
        need = size_t(D->red_w) * D->red_h * sizeof(float4);
        break;
    case AE_IMAGE_HISTORY_GEOMETRY:
        if (!D) return c->fail(AE_ERR_STATE, "no deferred frame yet");
        src = D->geom[D->history].ptr;
        need = px * sizeof(float4);
        break;
    case 100:  // deferred accumulation (accumTextures[historyIndex])
        if (!D) return c->fail(AE_ERR_STATE, "no deferred frame yet");
        src = D->accum[D->history].ptr;
        need = px * sizeof(float4);
        break;
    case 101: case 102: case 103: case 104: {  // G-buffer planes
        if (!D) return c->fail(AE_ERR_STATE, "no G-buffer yet");
        const void *pl[4] = {D->gpos.ptr, D->gnrm.ptr, D->galb.ptr, D->gdepth.ptr};
        const size_t sz[4] = {16, 16, 4, 4};
        src = pl[which - 101];
        need = px * sz[which - 101];
        break;
    }
    default:
        return c->fail(AE_ERR_INVALID, "unknown image %d", which);
    }
    if (bytes < need) return c->fail(AE_ERR_INVALID, "image needs %zu bytes, got %zu", need, bytes);
    int rc = c->cuda(cudaMemcpyAsync(dst, src, need, cudaMemcpyDeviceToHost, c->stream), "read image");
    if (rc) return rc;
    return c->cuda(cudaStreamSynchronize(c->stream), "read image");
}

}  // namespace ae

using namespace ae;

extern "C" int ae_build_gbuffer(ae_ctx *ctx) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c) return AE_ERR_INVALID;
    if (!c->scene_uploaded) return c->fail(AE_ERR_STATE, "G-buffer before ae_upload_scene");
    if (c->scene_has_ggx) return c->fail(AE_ERR_STATE, "the hybrid passes have no GGX metal");
    int rc = ensure(c);
    if (rc) return rc;
    Deferred &D = *c->deferred;
    const DefParams P = make_def_params(c);
    GBuf G{D.gpos.ptr, D.gnrm.ptr, D.galb.ptr, D.gdepth.ptr};
    dim3 grid((P.F.width + 15) / 16, (P.F.height + 7) / 8);
    k_gbuffer<<<grid, 128, 0, c->stream>>>(c->scene(), P, G);
    c->launches++;
    if ((rc = c->cuda(cudaGetLastError(), "G-buffer launch"))) return rc;
    D.have_gbuffer = true;
    return AE_OK;
}

// Any hit in [tnear, tmax] with deferred.comp's blocking rules (Occluded,
// deferred:1115-1171): glass and lights never block; meshes take the any-hit
// walk (OccludedMesh, deferred:812-854).  One thread per ray.
__global__ void __launch_bounds__(128) k_any_hit(DevScene S, const ae_ray *__restrict__ rays,
                                                 const float *__restrict__ tmax, uint32_t n, uint8_t *__restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const ae_ray r = rays[i];
    uint32_t seed = 1u;
    out[i] = occluded(S, mk(r.ox, r.oy, r.oz), mk(r.dx, r.dy, r.dz), r.time, r.tnear, tmax[i], seed) ? 1 : 0;
}

extern "C" int ae_any_hit(ae_ctx *ctx, const ae_ray *rays, const float *tmax, uint32_t n, uint8_t *out) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c) return AE_ERR_INVALID;
    if (n && (!rays || !tmax || !out)) return c->fail(AE_ERR_INVALID, "null ray, bound or output buffer");
    if (!c->scene_uploaded) return c->fail(AE_ERR_STATE, "any hit before ae_upload_scene");
    if (n == 0) return AE_OK;
    DevBuf<ae_ray> dr;
    DevBuf<float> dt;
    DevBuf<uint8_t> dout;
    if (dr.reserve(n) || dt.reserve(n) || dout.reserve(n)) return c->fail(AE_ERR_OOM, "any-hit buffers");
    int rc = c->cuda(cudaMemcpyAsync(dr.ptr, rays, size_t(n) * sizeof(ae_ray), cudaMemcpyHostToDevice, c->stream), "copy");
    if (!rc) rc = c->cuda(cudaMemcpyAsync(dt.ptr, tmax, size_t(n) * sizeof(float), cudaMemcpyHostToDevice, c->stream), "copy");
    if (rc) return rc;
    if ((rc = c->timed_begin())) return rc;
    k_any_hit<<<(n + 127) / 128, 128, 0, c->stream>>>(c->scene(), dr.ptr, dt.ptr, n, dout.ptr);
    if ((rc = c->cuda(cudaGetLastError(), "any-hit launch"))) return rc;
    if ((rc = c->timed_end())) return rc;
    rc = c->cuda(cudaMemcpyAsync(out, dout.ptr, n, cudaMemcpyDeviceToHost, c->stream), "copy");
    if (!rc) rc = c->cuda(cudaStreamSynchronize(c->stream), "any hit");
    return rc;
}
