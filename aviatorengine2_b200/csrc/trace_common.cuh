// trace_common.cuh - device-side scene view and the reference-order
// intersection and shading routines shared by the plain kernels.
//
// The plain kernels reproduce the reference's order of operations exactly
// (every multiply/add through ae_math.h's round-to-nearest intrinsics), which
// is what makes their hit IDs, t values and RNG-driven radiance comparable bit
// for bit with the oracle.  Memory is read with 16-byte vector loads through
// the read-only path; a record is fetched only in the parts a test needs.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/ae_b200.h"
#include "ae_math.h"

namespace ae {

#define AE_DEV __device__ __forceinline__

// Traversal stack depths.  The builder caps depth at 20 (scene/bvh.h:101), so
// a walk needs at most 21 slots per level; the reference sizes them 32 (TLAS,
// hybrid:30) and 24 (BLAS, hybrid:25).
constexpr int kTlasStack = 32;
constexpr int kBlasStack = 24;
constexpr float kFarStart = 1000000.0f;  // hybrid:869

// Touch counters of one ray, by the traffic formula of the roofline:
// TLAS nodes, object records, instance records, BLAS nodes, triangles, winners.
struct Touch {
    uint32_t tlas, objects, instances, blas, tris, winners;
    uint32_t rays;  // traversals started (TraverseBVH calls)
};

struct DevScene {
    const ae_object *objects;
    const ae_bvh_node *tlas;
    const uint32_t *lights;
    const ae_vertex *vertices;
    const uint32_t *indices;
    const ae_bvh_node *blas;
    const ae_instance *instances;
    uint32_t n_objects, n_nodes, n_lights, n_instances;
    // material texture array (RGBA8 sRGB words, layer-major) and the sRGB
    // decode table; tex_layers == 0: no array uploaded (samples white)
    const uint32_t *tex;
    const float *srgb;
    uint32_t tex_w, tex_h, tex_layers;
};

AE_DEV float4 ld4(const void *p) { return __ldg(reinterpret_cast<const float4 *>(p)); }

// A node's box and links, loaded as three 16-byte words.
struct NodeBox {
    f3 lo, hi;
    int left, right, count;
};
AE_DEV NodeBox load_node(const ae_bvh_node *nodes, uint32_t i) {
    const float4 *p = reinterpret_cast<const float4 *>(nodes + i);
    const float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
    NodeBox n;
    n.lo = mk(a.x, a.y, a.z);
    n.hi = mk(b.x, b.y, b.z);
    n.left = __float_as_int(b.w);
    n.right = __float_as_int(c.x);
    n.count = __float_as_int(c.y);
    return n;
}

// IntersectAABB, hybrid:547-562.
AE_DEV bool slab_ref(f3 o, f3 inv, f3 lo, f3 hi, float tn, float tf) {
    const f3 t0 = (lo - o) * inv;
    const f3 t1 = (hi - o) * inv;
    const f3 a = vmin(t0, t1), b = vmax(t0, t1);
    const float tmin = fmax_(fmax_(a.x, a.y), fmax_(a.z, tn));
    const float tmax = fmin_(fmin_(b.x, b.y), fmin_(b.z, tf));
    return tmin <= tmax;
}

// The fields of an object record the traversal and shading read.
struct ObjHead {  // bytes 112..127: refraction, shapeType, colorType, textureID
    float refraction;
    uint32_t shape, material, texture;
};
AE_DEV ObjHead load_head(const ae_object *o) {
    const float4 v = ld4(reinterpret_cast<const char *>(o) + 112);
    return ObjHead{v.x, __float_as_uint(v.y), __float_as_uint(v.z), __float_as_uint(v.w)};
}

// Closest-hit result kept by the device traversal.
struct DHit {
    float t;
    f3 p, n;
    bool front;
    uint32_t slot, prim;
    float alpha, beta;
};

// Watertight test: shear the triangle into the ray's frame and decide inside
// by the signs of the three 2D edge functions, falling back to double when an
// edge function is exactly zero (Woop, Benthin and Wald 2013, sections 3-4).
struct WtRay {
    int kx, ky, kz;
    float sx, sy, sz;
};
AE_DEV WtRay wt_setup(f3 d) {
    const float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    int kz = ax > ay ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
    int kx = kz == 2 ? 0 : kz + 1;
    int ky = kx == 2 ? 0 : kx + 1;
    const float dk[3] = {d.x, d.y, d.z};
    if (dk[kz] < 0.0f) { const int tmp = kx; kx = ky; ky = tmp; }
    WtRay w;
    w.kx = kx; w.ky = ky; w.kz = kz;
    w.sx = __fdiv_rn(dk[kx], dk[kz]);
    w.sy = __fdiv_rn(dk[ky], dk[kz]);
    w.sz = __fdiv_rn(1.0f, dk[kz]);
    return w;
}
AE_DEV float comp(f3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }
AE_DEV bool tri_wt(f3 o, const WtRay &W, float tn, float tf, f3 p0, f3 p1, f3 p2, float &t, float &a, float &b) {
    const f3 A = p0 - o, B = p1 - o, C = p2 - o;
    const float Az = comp(A, W.kz), Bz = comp(B, W.kz), Cz = comp(C, W.kz);
    const float Ax = __fsub_rn(comp(A, W.kx), __fmul_rn(W.sx, Az)), Ay = __fsub_rn(comp(A, W.ky), __fmul_rn(W.sy, Az));
    const float Bx = __fsub_rn(comp(B, W.kx), __fmul_rn(W.sx, Bz)), By = __fsub_rn(comp(B, W.ky), __fmul_rn(W.sy, Bz));
    const float Cx = __fsub_rn(comp(C, W.kx), __fmul_rn(W.sx, Cz)), Cy = __fsub_rn(comp(C, W.ky), __fmul_rn(W.sy, Cz));
    float U = __fsub_rn(__fmul_rn(Cx, By), __fmul_rn(Cy, Bx));
    float V = __fsub_rn(__fmul_rn(Ax, Cy), __fmul_rn(Ay, Cx));
    float Wv = __fsub_rn(__fmul_rn(Bx, Ay), __fmul_rn(By, Ax));
    if (U == 0.0f || V == 0.0f || Wv == 0.0f) {
        U = float(double(Cx) * double(By) - double(Cy) * double(Bx));
        V = float(double(Ax) * double(Cy) - double(Ay) * double(Cx));
        Wv = float(double(Bx) * double(Ay) - double(By) * double(Ax));
    }
    if ((U < 0.0f || V < 0.0f || Wv < 0.0f) && (U > 0.0f || V > 0.0f || Wv > 0.0f)) return false;
    const float det = __fadd_rn(__fadd_rn(U, V), Wv);
    if (det == 0.0f) return false;
    const float T = __fadd_rn(__fadd_rn(__fmul_rn(U, __fmul_rn(W.sz, Az)), __fmul_rn(V, __fmul_rn(W.sz, Bz))),
                              __fmul_rn(Wv, __fmul_rn(W.sz, Cz)));
    t = __fdiv_rn(T, det);
    if (!(t >= tn) || t > tf) return false;
    a = __fdiv_rn(V, det);
    b = __fdiv_rn(Wv, det);
    return true;
}

// HitMeshTriangle, hybrid:564-598.
AE_DEV bool tri_ref(f3 o, f3 d, float tn, float tf, f3 p0, f3 p1, f3 p2, float &t, float &a, float &b, f3 &geo) {
    const f3 e1 = p1 - p0, e2 = p2 - p0;
    const f3 n = cross(e1, e2);
    const float nn = dot(n, n);
    if (nn < 1e-12f) return false;
    const float den = dot(n, d);
    if (AE_FABS(den) < 1e-12f) return false;
    t = AE_DIV(AE_SUB(dot(n, p0), dot(n, o)), den);
    if (t < tn || t > tf) return false;
    const f3 w = n / nn;
    const f3 pl = o + d * t - p0;
    a = dot(w, cross(pl, e2));
    b = dot(w, cross(e1, pl));
    if (a < 0.0f || b < 0.0f || AE_ADD(a, b) > 1.0f) return false;
    geo = n / AE_SQRT(nn);
    return true;
}

// Debug checks of the reference walk (AE_VARIANT_PLAIN_CHECKED): every stack
// push against the stack's capacity and every buffer index against its
// array's length.  A violation skips the access - a node not visited, a
// triangle or object not tested - and sets its bit (AE_CHECK_STACK,
// AE_CHECK_INDEX) in *flags.  Passed as a null pointer, as by every other
// caller, the checks compile away.
struct Checks {
    uint32_t *flags;
    uint32_t n_nodes, n_objects, n_instances, n_blas, n_indices, n_vertices;
    int tlas_stack, blas_stack;  // capacities checked (at most kTlasStack, kBlasStack)
};
AE_DEV void check_fail(const Checks *ck, uint32_t bit) { atomicOr(ck->flags, bit); }

AE_DEV f3 vtx_pos(const ae_vertex *v, uint32_t i) {
    const float4 a = ld4(v + i);
    return mk(a.x, a.y, a.z);
}

// HitMesh, hybrid:600-707 (ToLocal hybrid:534-543; pad0 scale extension).
// WT = true swaps HitMeshTriangle for the watertight test above and keeps
// everything else, visit order and tie rule included: the FP32-node form of
// the precision variant's triangle test.
template <bool WT = false>
AE_DEV bool hit_mesh_ref(const DevScene &S, uint32_t inst_index, f3 o, f3 d, float tn, float tf, DHit &h,
                         Touch *T = nullptr, const Checks *CK = nullptr) {
    if (T) T->instances++;
    if (CK && inst_index >= CK->n_instances) {
        check_fail(CK, AE_CHECK_INDEX);
        return false;
    }
    const float4 *ip = reinterpret_cast<const float4 *>(S.instances + inst_index);
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
    WtRay W;
    if (WT) W = wt_setup(ld);
    int stack[kBlasStack];
    int sp = 0;
    stack[sp++] = 0;
    bool found = false;
    float closest = tf, ba = 0.0f, bb = 0.0f;
    uint32_t best = 0;
    f3 bgeo = mk(0.0f, 0.0f, 1.0f);
    while (sp > 0) {
        const uint32_t ni = bbase + uint32_t(stack[--sp]);
        if (CK && ni >= CK->n_blas) {
            check_fail(CK, AE_CHECK_INDEX);
            continue;
        }
        const NodeBox n = load_node(S.blas, ni);
        if (T) T->blas++;
        if (!slab_ref(lo, invd, n.lo, n.hi, tn, closest)) continue;
        if (n.count > 0) {
            for (int i = 0; i < n.count; ++i) {
                const uint32_t base = ibase + uint32_t(n.left + i) * 3u;
                if (T) T->tris++;
                if (CK && base + 2u >= CK->n_indices) {
                    check_fail(CK, AE_CHECK_INDEX);
                    continue;
                }
                const uint32_t a0 = __ldg(S.indices + base), a1 = __ldg(S.indices + base + 1),
                               a2 = __ldg(S.indices + base + 2);
                if (CK && (vbase + a0 >= CK->n_vertices || vbase + a1 >= CK->n_vertices ||
                          vbase + a2 >= CK->n_vertices)) {
                    check_fail(CK, AE_CHECK_INDEX);
                    continue;
                }
                const f3 p0 = vtx_pos(S.vertices, vbase + a0), p1 = vtx_pos(S.vertices, vbase + a1),
                         p2 = vtx_pos(S.vertices, vbase + a2);
                float t, a, b;
                f3 g;
                const bool hit = WT ? tri_wt(lo, W, tn, closest, p0, p1, p2, t, a, b)
                                    : tri_ref(lo, ld, tn, closest, p0, p1, p2, t, a, b, g);
                if (hit) {
                    closest = t; found = true; ba = a; bb = b; best = base;
                    if (!WT) bgeo = g;
                }
            }
        } else if (sp + 2 <= (CK ? CK->blas_stack : kBlasStack)) {
            stack[sp++] = n.left;
            stack[sp++] = n.right;
        } else if (CK) {
            check_fail(CK, AE_CHECK_STACK);
        }
    }
    if (!found) return false;
    if (T) T->winners++;
    const ae_vertex *A = S.vertices + vbase + __ldg(S.indices + best);
    const ae_vertex *B = S.vertices + vbase + __ldg(S.indices + best + 1);
    const ae_vertex *C = S.vertices + vbase + __ldg(S.indices + best + 2);
    const float4 a1 = ld4(reinterpret_cast<const char *>(A) + 16), b1 = ld4(reinterpret_cast<const char *>(B) + 16),
                 c1 = ld4(reinterpret_cast<const char *>(C) + 16);
    const float4 a0 = ld4(A), b0 = ld4(B), c0 = ld4(C);
    if (WT) {
        const f3 n = cross(mk(b0.x, b0.y, b0.z) - mk(a0.x, a0.y, a0.z), mk(c0.x, c0.y, c0.z) - mk(a0.x, a0.y, a0.z));
        bgeo = n / AE_SQRT(dot(n, n));
    }
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

// HitQuad (hybrid:425-478) and HitTriangle (hybrid:480-513).
AE_DEV bool hit_planar_ref(const ae_object *obj, bool tri, f3 o, f3 d, float tn, float tf, DHit &h) {
    const char *base = reinterpret_cast<const char *>(obj);
    const float4 q0 = ld4(base), q2 = ld4(base + 32), q3 = ld4(base + 48);
    const f3 P = mk(q0.x, q0.y, q0.z), U = mk(q2.x, q2.y, q2.z), W = mk(q3.x, q3.y, q3.z);
    const f3 n = cross(U, W);
    const float nn = dot(n, n);
    if (nn < 1e-8f) return false;
    const f3 unit = n / AE_SQRT(nn);
    const f3 w = n / nn;
    const float den = dot(n, d);
    if (AE_FABS(den) < 1e-8f) return false;
    const float t = AE_DIV(AE_SUB(dot(n, P), dot(n, o)), den);
    if (t < tn || t > tf) return false;
    const f3 X = o + d * t;
    const f3 pl = X - P;
    const float a = dot(w, cross(pl, W));
    const float b = dot(w, cross(U, pl));
    if (!tri) {
        if (a < 0.0f || a > 1.0f || b < 0.0f || b > 1.0f) return false;
    } else if (a < 0.0f || b < 0.0f || AE_ADD(a, b) > 1.0f) {
        return false;
    }
    h.t = t;
    h.p = X;
    h.n = unit;
    h.front = dot(d, unit) < 0.0f;
    if (!h.front) h.n = -h.n;
    h.alpha = a;
    h.beta = b;
    h.prim = AE_MISS;
    return true;
}

// SphereSpan + HitSphere, hybrid:285-297, 382-423.
AE_DEV bool hit_sphere_ref(const ae_object *obj, f3 o, f3 d, float time, float tn, float tf, DHit &h) {
    const char *base = reinterpret_cast<const char *>(obj);
    const float4 q0 = ld4(base), q1 = ld4(base + 16);
    const f3 P = mk(q0.x, q0.y, q0.z), P2 = mk(q1.x, q1.y, q1.z);
    const float radius = q1.w;
    const f3 c = lerp(P, P2, time);
    const f3 oc = c - o;
    const float a = dot(d, d), b = dot(d, oc);
    const float cc = AE_SUB(dot(oc, oc), AE_MUL(radius, radius));
    const float disc = AE_SUB(AE_MUL(b, b), AE_MUL(a, cc));
    if (disc < 0.0f) return false;
    const float sq = AE_SQRT(disc);
    float root = AE_DIV(AE_SUB(b, sq), a);
    if (root <= tn || tf <= root) {
        root = AE_DIV(AE_ADD(b, sq), a);
        if (root <= tn || tf <= root) return false;
    }
    h.t = root;
    h.p = o + d * root;
    h.n = (h.p - c) / radius;
    h.front = dot(d, h.n) < 0.0f;
    if (!h.front) h.n = -h.n;
    h.alpha = 0.0f;
    h.beta = 0.0f;
    h.prim = AE_MISS;
    return true;
}

// BoxIntersect + HitBox, hybrid:315-348, 729-773 (face UVs are not needed by
// any consumer of the device hit).
AE_DEV f3 yaw_rot(f3 v, float s, float c) {
    return mk(AE_ADD(AE_MUL(c, v.x), AE_MUL(s, v.z)), v.y, AE_ADD(AE_MUL(-s, v.x), AE_MUL(c, v.z)));
}
AE_DEV bool box_span_ref(const ae_object *obj, f3 o, f3 d, float &tin, float &tout, f3 &nin, f3 &nout) {
    const char *base = reinterpret_cast<const char *>(obj);
    const float4 q0 = ld4(base), q4 = ld4(base + 64);
    const float s = sinf_(q4.w), c = cosf_(q4.w);
    const f3 lo = yaw_rot(o - mk(q0.x, q0.y, q0.z), -s, c);
    const f3 ld = yaw_rot(d, -s, c);
    const f3 inv = 1.0f / ld;
    const f3 he = mk(q4.x, q4.y, q4.z);
    const f3 t0 = (-he - lo) * inv, t1 = (he - lo) * inv;
    const f3 a = vmin(t0, t1), b = vmax(t0, t1);
    tin = fmax_(fmax_(a.x, a.y), a.z);
    tout = fmin_(fmin_(b.x, b.y), b.z);
    nin = mk(0.0f, 0.0f, -signf(ld.z));
    if (tin == a.x) nin = mk(-signf(ld.x), 0.0f, 0.0f);
    else if (tin == a.y) nin = mk(0.0f, -signf(ld.y), 0.0f);
    nout = mk(0.0f, 0.0f, signf(ld.z));
    if (tout == b.x) nout = mk(signf(ld.x), 0.0f, 0.0f);
    else if (tout == b.y) nout = mk(0.0f, signf(ld.y), 0.0f);
    return tout > tin;
}
AE_DEV bool hit_box_ref(const ae_object *obj, f3 o, f3 d, float tn, float tf, DHit &h) {
    float tin, tout;
    f3 nin, nout;
    if (!box_span_ref(obj, o, d, tin, tout, nin, nout)) return false;
    float t = tin;
    f3 ln = nin;
    bool outside = true;
    if (t <= tn || tf <= t) {
        t = tout; ln = nout; outside = false;
        if (t <= tn || tf <= t) return false;
    }
    const float rot = ld4(reinterpret_cast<const char *>(obj) + 64).w;
    h.t = t;
    h.p = o + d * t;
    h.n = yaw_rot(ln, sinf_(rot), cosf_(rot));
    h.front = outside;
    if (!h.front) h.n = -h.n;
    h.alpha = 0.0f;
    h.beta = 0.0f;
    h.prim = AE_MISS;
    return true;
}

// HitVolume, hybrid:779-822 (one RNG draw).
AE_DEV bool hit_volume_ref(const ae_object *obj, uint32_t shape, f3 o, f3 d, float time, float tn, float tf,
                           DHit &h, uint32_t &seed) {
    float a, b;
    if (shape == AE_SHAPE_SPHERE) {
        DHit tmp;
        // SphereSpan roots without the window test.
        const char *base = reinterpret_cast<const char *>(obj);
        const float4 q0 = ld4(base), q1 = ld4(base + 16);
        const f3 c = lerp(mk(q0.x, q0.y, q0.z), mk(q1.x, q1.y, q1.z), time);
        const f3 oc = c - o;
        const float aa = dot(d, d), bb = dot(d, oc);
        const float cc = AE_SUB(dot(oc, oc), AE_MUL(q1.w, q1.w));
        const float disc = AE_SUB(AE_MUL(bb, bb), AE_MUL(aa, cc));
        (void)tmp;
        if (disc < 0.0f) return false;
        const float sq = AE_SQRT(disc);
        a = AE_DIV(AE_SUB(bb, sq), aa);
        b = AE_DIV(AE_ADD(bb, sq), aa);
    } else if (shape == AE_SHAPE_BOX) {
        f3 n0, n1;
        if (!box_span_ref(obj, o, d, a, b, n0, n1)) return false;
    } else {
        return false;
    }
    a = fmax_(a, tn);
    b = fmin_(b, tf);
    if (a >= b) return false;
    const float rl = length(d);
    const float inside = AE_MUL(AE_SUB(b, a), rl);
    const float density = ld4(reinterpret_cast<const char *>(obj) + 80).x;
    const float dist = AE_DIV(-logf_(fmax_(rng_next(seed), 1e-8f)), fmax_(density, 1e-8f));
    if (dist > inside) return false;
    h.t = AE_ADD(a, AE_DIV(dist, rl));
    h.p = o + d * h.t;
    h.n = mk(0.0f, 1.0f, 0.0f);
    h.front = true;
    h.alpha = 0.0f;
    h.beta = 0.0f;
    h.prim = AE_MISS;
    return true;
}

// TraverseBVH, hybrid:862-917, and HitObject dispatch, hybrid:827-856.
// WT selects the watertight triangle test inside meshes (hit_mesh_ref).
template <bool WT = false>
AE_DEV bool traverse_ref(const DevScene &S, f3 o, f3 d, float time, float tn, DHit &out, uint32_t &seed,
                         Touch *T = nullptr, const Checks *CK = nullptr) {
    if (T) T->rays++;
    if (S.n_nodes == 0) return false;
    const f3 inv = 1.0f / d;
    int stack[kTlasStack];
    int sp = 0;
    stack[sp++] = 0;
    bool found = false;
    float tf = kFarStart;
    while (sp > 0) {
        const uint32_t ni = uint32_t(stack[--sp]);
        if (CK && ni >= CK->n_nodes) {
            check_fail(CK, AE_CHECK_INDEX);
            continue;
        }
        const NodeBox n = load_node(S.tlas, ni);
        if (T) T->tlas++;
        if (!slab_ref(o, inv, n.lo, n.hi, tn, tf)) continue;
        if (n.count > 0) {
            for (int i = 0; i < n.count; i++) {
                const uint32_t slot = uint32_t(n.left + i);
                if (CK && slot >= CK->n_objects) {
                    check_fail(CK, AE_CHECK_INDEX);
                    continue;
                }
                const ae_object *obj = S.objects + slot;
                if (T) T->objects++;
                const ObjHead hd = load_head(obj);
                DHit h;
                bool hit;
                if (hd.material == AE_MAT_ISOTROPIC) hit = hit_volume_ref(obj, hd.shape, o, d, time, tn, tf, h, seed);
                else if (hd.shape == AE_SHAPE_SPHERE) hit = hit_sphere_ref(obj, o, d, time, tn, tf, h);
                else if (hd.shape == AE_SHAPE_QUAD) hit = hit_planar_ref(obj, false, o, d, tn, tf, h);
                else if (hd.shape == AE_SHAPE_TRIANGLE) hit = hit_planar_ref(obj, true, o, d, tn, tf, h);
                else if (hd.shape == AE_SHAPE_MESH) {
                    const uint32_t inst = __float_as_uint(ld4(reinterpret_cast<const char *>(obj) + 80).z);
                    hit = hit_mesh_ref<WT>(S, inst, o, d, tn, tf, h, T, CK);
                } else hit = hit_box_ref(obj, o, d, tn, tf, h);
                if (hit) {
                    tf = h.t;
                    h.slot = slot;
                    out = h;
                    found = true;
                }
            }
        } else if (sp + 2 <= (CK ? CK->tlas_stack : kTlasStack)) {
            stack[sp++] = n.left;
            stack[sp++] = n.right;
        } else if (CK) {
            check_fail(CK, AE_CHECK_STACK);
        }
    }
    return found;
}

}  // namespace ae
