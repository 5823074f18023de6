// shade.cuh - device-side shading shared by the plain megakernel and the
// wavefront path tracer: materials, light sampling, bounces (restating
// shaders/ray_trace.comp.hybrid.hlsl, `hybrid:N`), camera rays, and the
// reconstruction of a hit's surface from a closest-hit record.  Every
// operation goes through ae_math.h, so both forms produce identical bits.
#pragma once
#include "kernels.h"
#include "trace_common.cuh"

namespace ae {

struct MatRec {
    f3 albedo;
    float fuzz, emission, refraction;
    uint32_t type;
    uint32_t texture;  // layer in the texture array, or AE_NO_TEXTURE
    float tint;        // TextureTint
};
AE_DEV MatRec load_mat(const ae_object *o) {
    const char *b = reinterpret_cast<const char *>(o);
    const float4 m0 = ld4(b + 80), m1 = ld4(b + 96), m2 = ld4(b + 112);
    return MatRec{mk(m1.x, m1.y, m1.z), m1.w, m0.y, m2.x, __float_as_uint(m2.z), __float_as_uint(m2.w), m0.w};
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
// T (optional): touch counters of the shadow traversals.
AE_DEV f3 direct_light(const DevScene &S, const DHit &h, f3 surf_albedo, float time, uint32_t &seed,
                       Touch *T = nullptr) {
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
            if (!traverse_ref(S, so, sd, time, 0.001f, sh, seed, T)) break;
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

// Rough metal with GGX microfacet reflection - an extension: the
// reference's METAL is a mirror blurred by fuzz (hybrid:988-991).  The model
// is Walter, Marschner, Li and Torrance, "Microfacet Models for Refraction
// through Rough Surfaces" (EGSR 2007), with alpha = the material's roughness
// (Object_GPU::fuzz):
//   * a microfacet normal m drawn with density D(m)|m.n| (eqs. 35-36):
//     cos^2(theta_m) = (1 - u1) / (1 + (alpha^2 - 1) u1), phi_m = 2 pi u2,
//     placed in an orthonormal basis around n (Duff et al., "Building an
//     Orthonormal Basis, Revisited", JCGT 2017);
//   * the mirror direction o = 2 (i.m) m - i about m (eq. 39), i = -d;
//   * the sample weight F(i.m) |i.m| G(i,o,m) / (|i.n| |m.n|) (eq. 41), with
//     the Smith shadowing G = G1(i) G1(o), G1(v) = 2 / (1 + sqrt(1 + alpha^2
//     tan^2 theta_v)) (eq. 34), and Schlick's Fresnel with F0 = albedo.
// Two RNG draws, always taken.  Returns false when the path ends (i or o
// below the shading surface).
AE_DEV float ggx_g1(float cv, float a2) {
    const float c2 = AE_MUL(cv, cv);
    const float t2 = AE_DIV(AE_SUB(1.0f, c2), c2);
    return AE_DIV(2.0f, AE_ADD(1.0f, AE_SQRT(AE_ADD(1.0f, AE_MUL(a2, t2)))));
}
AE_DEV bool ggx_bounce(f3 d, f3 n, f3 albedo, float alpha, f3 &dir, f3 &weight, uint32_t &seed) {
    const f3 i = -normalize(d);
    const float u1 = rng_next(seed);
    const float u2 = rng_next(seed);
    const float cin = dot(i, n);
    if (cin <= 0.0f) return false;
    const float a2 = AE_MUL(alpha, alpha);
    const float c2 = AE_DIV(AE_SUB(1.0f, u1), AE_ADD(1.0f, AE_MUL(AE_SUB(a2, 1.0f), u1)));
    const float cm = AE_SQRT(c2);
    const float sm = AE_SQRT(fmax_(0.0f, AE_SUB(1.0f, c2)));
    const float phi = AE_MUL(6.2831853f, u2);
    const float cp = cosf_(phi), sp = sinf_(phi);
    const float sg = n.z >= 0.0f ? 1.0f : -1.0f;
    const float a = AE_DIV(-1.0f, AE_ADD(sg, n.z));
    const float b = AE_MUL(AE_MUL(n.x, n.y), a);
    const f3 t = mk(AE_ADD(1.0f, AE_MUL(AE_MUL(sg, AE_MUL(n.x, n.x)), a)), AE_MUL(sg, b), -AE_MUL(sg, n.x));
    const f3 bt = mk(b, AE_ADD(sg, AE_MUL(AE_MUL(n.y, n.y), a)), -n.y);
    const f3 m = t * AE_MUL(sm, cp) + bt * AE_MUL(sm, sp) + n * cm;
    const float im = dot(i, m);
    if (im <= 0.0f) return false;
    dir = m * AE_MUL(2.0f, im) - i;
    const float con = dot(dir, n);
    if (con <= 0.0f) return false;
    const float g = AE_MUL(ggx_g1(cin, a2), ggx_g1(con, a2));
    const float w = AE_DIV(AE_MUL(im, g), AE_MUL(cin, cm));
    const float f5 = powf_(AE_SUB(1.0f, im), 5.0f);
    const f3 fr = albedo + (splat(1.0f) - albedo) * f5;
    weight = fr * w;
    return true;
}

// GetBounce, hybrid:965-1033, and the GGX metal extension above.  `alb` is
// the surface albedo (GGX's F0); `ggx_w` receives the GGX sample weight,
// which replaces the albedo in the throughput update for that material.
AE_DEV bool get_bounce(f3 d, const DHit &h, const MatRec &m, f3 alb, f3 &dir, f3 &ggx_w, uint32_t &seed) {
    dir = splat(0.0f);
    switch (m.type) {
    case AE_MAT_GGX_METAL:
        return ggx_bounce(d, h.n, alb, m.fuzz, dir, ggx_w, seed);
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

// One camera sample of pixel (x, y) drawn from the pixel's running RNG state:
// jitter, defocus, direction and time (hybrid:1366-1373).
AE_DEV void camera_sample(const FrameParams &F, uint32_t x, uint32_t y, f3 &o, f3 &d, float &time, uint32_t &seed) {
    const float jx = AE_SUB(rng_next(seed), 0.5f);
    const float jy = AE_SUB(rng_next(seed), 0.5f);
    const f3 tgt = F.pixel0 + AE_ADD(AE_U2F(x), jx) * F.pixel_u + AE_ADD(AE_U2F(y), jy) * F.pixel_v;
    o = F.source;
    if (F.defocus_angle > 0.0f) {
        float px, py;
        for (;;) {
            const float a = rng_next(seed), b = rng_next(seed);
            px = AE_SUB(AE_MUL(a, 2.0f), 1.0f);
            py = AE_SUB(AE_MUL(b, 2.0f), 1.0f);
            if (length(mk(px, py, 0.0f)) < 1.0f) break;
        }
        o = F.source + px * F.defocus_u + py * F.defocus_v;
    }
    d = normalize(tgt - o);
    time = rng_next(seed);
}

// The first sample of a frame: the per-pixel seed, then camera_sample.
AE_DEV void camera_ray(const FrameParams &F, uint32_t x, uint32_t y, f3 &o, f3 &d, float &time, uint32_t &seed) {
    seed = x + y * F.width + F.batch * F.width * F.height + 1u;
    camera_sample(F, x, y, o, d, time, seed);
}

// World shading normal and facing of a mesh hit, recomputed from the hit
// record exactly as HitMesh finishes (hybrid:655-706).
AE_DEV bool hit_normal(const DevScene &S, const ae_hit &h, f3 d, f3 &n) {
    if (h.object == AE_MISS) return false;
    const ae_object *obj = S.objects + h.object;
    const ObjHead hd = load_head(obj);
    if (hd.shape != AE_SHAPE_MESH) {
        // Planar objects: the unit plane normal facing the ray.
        const char *b = reinterpret_cast<const char *>(obj);
        const float4 q2 = ld4(b + 32), q3 = ld4(b + 48);
        const f3 nn = cross(mk(q2.x, q2.y, q2.z), mk(q3.x, q3.y, q3.z));
        n = nn / AE_SQRT(dot(nn, nn));
        if (!(dot(d, n) < 0.0f)) n = -n;
        return hd.shape == AE_SHAPE_QUAD || hd.shape == AE_SHAPE_TRIANGLE;
    }
    const uint32_t ii = __float_as_uint(ld4(reinterpret_cast<const char *>(obj) + 80).z);
    const float4 *ip = reinterpret_cast<const float4 *>(S.instances + ii);
    const float4 i1 = __ldg(ip + 1), i2 = __ldg(ip + 2);
    const uint32_t vbase = __float_as_uint(i2.x), ibase = __float_as_uint(i2.y);
    const uint32_t base = ibase + h.prim * 3u;
    const ae_vertex *A = S.vertices + vbase + __ldg(S.indices + base);
    const ae_vertex *B = S.vertices + vbase + __ldg(S.indices + base + 1);
    const ae_vertex *C = S.vertices + vbase + __ldg(S.indices + base + 2);
    const float4 a0 = ld4(A), b0 = ld4(B), c0 = ld4(C);
    const float4 a1 = ld4(reinterpret_cast<const char *>(A) + 16), b1 = ld4(reinterpret_cast<const char *>(B) + 16),
                 c1 = ld4(reinterpret_cast<const char *>(C) + 16);
    const float w0 = AE_SUB(AE_SUB(1.0f, h.alpha), h.beta);
    const f3 sh = normalize(w0 * mk(a0.w, a1.x, a1.y) + h.alpha * mk(b0.w, b1.x, b1.y) + h.beta * mk(c0.w, c1.x, c1.y));
    const f3 p0 = mk(a0.x, a0.y, a0.z);
    const f3 gn = cross(mk(b0.x, b0.y, b0.z) - p0, mk(c0.x, c0.y, c0.z) - p0);
    f3 geo = gn / AE_SQRT(dot(gn, gn));
    if (dot(geo, sh) < 0.0f) geo = -geo;
    n = normalize(quat_rotate(i1.x, i1.y, i1.z, i1.w, sh));
    if (!(dot(d, quat_rotate(i1.x, i1.y, i1.z, i1.w, geo)) < 0.0f)) n = -n;
    return true;
}

// Surface UV of a hit, recomputed from its record exactly as the intersector
// that produced it sets hit.surface_uv: meshes interpolate the vertex UVs
// (hybrid:702-704), quads and triangles take (alpha, beta) (467, 505),
// spheres get_sphere_uv of the facing normal (264-271, 419), boxes BoxFaceUV
// of the local hit point (711-727, 763), volumes (0, 0) (819).
AE_DEV void hit_uv(const DevScene &S, const DHit &h, f3 o, f3 d, float &u, float &v) {
    const ae_object *obj = S.objects + h.slot;
    const ObjHead hd = load_head(obj);
    const char *b = reinterpret_cast<const char *>(obj);
    u = 0.0f;
    v = 0.0f;
    if (hd.material == AE_MAT_ISOTROPIC) return;
    if (hd.shape == AE_SHAPE_MESH) {
        const uint32_t ii = __float_as_uint(ld4(b + 80).z);
        const float4 i2 = ld4(reinterpret_cast<const char *>(S.instances + ii) + 32);
        const uint32_t vbase = __float_as_uint(i2.x), base = __float_as_uint(i2.y) + h.prim * 3u;
        const float4 a1 = ld4(reinterpret_cast<const char *>(S.vertices + vbase + __ldg(S.indices + base)) + 16);
        const float4 b1 = ld4(reinterpret_cast<const char *>(S.vertices + vbase + __ldg(S.indices + base + 1)) + 16);
        const float4 c1 = ld4(reinterpret_cast<const char *>(S.vertices + vbase + __ldg(S.indices + base + 2)) + 16);
        const float w0 = AE_SUB(AE_SUB(1.0f, h.alpha), h.beta);
        u = AE_ADD(AE_ADD(AE_MUL(w0, a1.z), AE_MUL(h.alpha, b1.z)), AE_MUL(h.beta, c1.z));
        v = AE_ADD(AE_ADD(AE_MUL(w0, a1.w), AE_MUL(h.alpha, b1.w)), AE_MUL(h.beta, c1.w));
        return;
    }
    if (hd.shape == AE_SHAPE_QUAD || hd.shape == AE_SHAPE_TRIANGLE) {
        u = h.alpha;
        v = h.beta;
        return;
    }
    if (hd.shape == AE_SHAPE_SPHERE) {
        const float rot = ld4(b + 64).w;
        const float theta = acosf_(-h.n.y);
        const float phi = AE_ADD(atan2f_(-h.n.z, h.n.x), 3.14159265f);
        u = fracf(AE_SUB(AE_DIV(phi, 6.2831853f), AE_DIV(rot, 6.2831853f)));
        v = AE_DIV(theta, 3.14159265f);
        return;
    }
    // Box: the local ray of BoxSpan, the face it was hit on.
    const float4 q0 = ld4(b), q4 = ld4(b + 64);
    const float sn = sinf_(q4.w), cs = cosf_(q4.w);
    const f3 lo = yaw_rot(o - mk(q0.x, q0.y, q0.z), -sn, cs);
    const f3 ld = yaw_rot(d, -sn, cs);
    float tin, tout;
    f3 nin, nout;
    box_span_ref(obj, o, d, tin, tout, nin, nout);
    const f3 ln = h.t == tin ? nin : nout;
    const f3 lp = lo + ld * h.t;
    float uu, vv;
    if (AE_FABS(ln.x) > 0.5f) { uu = AE_DIV(lp.z, q4.z); vv = AE_DIV(lp.y, q4.y); }
    else if (AE_FABS(ln.y) > 0.5f) { uu = AE_DIV(lp.x, q4.x); vv = AE_DIV(lp.z, q4.z); }
    else { uu = AE_DIV(lp.x, q4.x); vv = AE_DIV(lp.y, q4.y); }
    u = saturate(AE_ADD(AE_MUL(uu, 0.5f), 0.5f));
    v = saturate(AE_ADD(AE_MUL(vv, 0.5f), 0.5f));
}

// SurfaceAlbedo, hybrid:940-949: the flat albedo, or the texel at the hit's
// UV tinted by the albedo (texel * lerp(1, albedo, TextureTint)).
AE_DEV f3 surface_albedo(const DevScene &S, const DHit &h, const MatRec &m, f3 o, f3 d) {
    if (m.texture == AE_NO_TEXTURE) return m.albedo;
    float u, v;
    hit_uv(S, h, o, d, u, v);
    const f3 texel = texture_sample(S.tex, S.srgb, S.tex_w, S.tex_h, S.tex_layers, m.texture, u, v);
    return texel * lerp(splat(1.0f), m.albedo, m.tint);
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

// The surface of a closest hit - position, facing normal, facing flag -
// recomputed from its record exactly as the intersector that produced it
// finishes (HitQuad hybrid:467-476, HitSphere 407-422, HitBox 752-772,
// HitMesh 655-706).  Returns false on a miss.
AE_DEV bool surface_from_hit(const DevScene &S, const ae_hit &h, f3 o, f3 d, float time, DHit &out) {
    if (h.object == AE_MISS) return false;
    const ae_object *obj = S.objects + h.object;
    const ObjHead hd = load_head(obj);
    const char *b = reinterpret_cast<const char *>(obj);
    out.t = h.t;
    out.slot = h.object;
    out.prim = h.prim;
    out.alpha = h.alpha;
    out.beta = h.beta;
    out.p = o + d * h.t;
    if (hd.shape == AE_SHAPE_MESH) {
        f3 n;
        hit_normal(S, h, d, n);
        out.n = n;
        // Facing as HitMesh decides it: by the geometric normal.
        const uint32_t ii = __float_as_uint(ld4(b + 80).z);
        const float4 q = ld4(reinterpret_cast<const char *>(S.instances + ii) + 16);
        const float4 i2 = ld4(reinterpret_cast<const char *>(S.instances + ii) + 32);
        const uint32_t vbase = __float_as_uint(i2.x), ibase = __float_as_uint(i2.y);
        const uint32_t base = ibase + h.prim * 3u;
        const f3 p0 = vtx_pos(S.vertices, vbase + __ldg(S.indices + base));
        const f3 p1 = vtx_pos(S.vertices, vbase + __ldg(S.indices + base + 1));
        const f3 p2 = vtx_pos(S.vertices, vbase + __ldg(S.indices + base + 2));
        const ae_vertex *A = S.vertices + vbase + __ldg(S.indices + base);
        const ae_vertex *B = S.vertices + vbase + __ldg(S.indices + base + 1);
        const ae_vertex *C = S.vertices + vbase + __ldg(S.indices + base + 2);
        const float4 a0 = ld4(A), b0 = ld4(B), c0 = ld4(C);
        const float4 a1 = ld4(reinterpret_cast<const char *>(A) + 16), b1 = ld4(reinterpret_cast<const char *>(B) + 16),
                     c1 = ld4(reinterpret_cast<const char *>(C) + 16);
        const float w0 = AE_SUB(AE_SUB(1.0f, h.alpha), h.beta);
        const f3 sh = normalize(w0 * mk(a0.w, a1.x, a1.y) + h.alpha * mk(b0.w, b1.x, b1.y) + h.beta * mk(c0.w, c1.x, c1.y));
        const f3 gn = cross(p1 - p0, p2 - p0);
        f3 geo = gn / AE_SQRT(dot(gn, gn));
        if (dot(geo, sh) < 0.0f) geo = -geo;
        out.front = dot(d, quat_rotate(q.x, q.y, q.z, q.w, geo)) < 0.0f;
        return true;
    }
    if (hd.shape == AE_SHAPE_QUAD || hd.shape == AE_SHAPE_TRIANGLE) {
        const float4 q2 = ld4(b + 32), q3 = ld4(b + 48);
        const f3 n = cross(mk(q2.x, q2.y, q2.z), mk(q3.x, q3.y, q3.z));
        out.n = n / AE_SQRT(dot(n, n));
        out.front = dot(d, out.n) < 0.0f;
        if (!out.front) out.n = -out.n;
        return true;
    }
    if (hd.shape == AE_SHAPE_SPHERE) {
        const float4 q0 = ld4(b), q1 = ld4(b + 16);
        const f3 c = lerp(mk(q0.x, q0.y, q0.z), mk(q1.x, q1.y, q1.z), time);
        out.n = (out.p - c) / q1.w;
        out.front = dot(d, out.n) < 0.0f;
        if (!out.front) out.n = -out.n;
        return true;
    }
    float tin, tout;
    f3 nin, nout;
    box_span_ref(obj, o, d, tin, tout, nin, nout);
    const bool outside = h.t == tin;
    const float rot = ld4(b + 64).w;
    out.n = yaw_rot(outside ? nin : nout, sinf_(rot), cosf_(rot));
    out.front = outside;
    if (!out.front) out.n = -out.n;
    return true;
}

}  // namespace ae
