// oracle.cpp - TEST INFRASTRUCTURE ONLY.  A CPU restatement of AviatorEngine2's
// ray/path-tracing hot path, used by tests/ as the parity checker and by
// bench.py as the timed CPU baseline.  The library never links or calls it.
//
// Parity pinning: the reference has no CPU ray tracer and no golden vectors
// for this path.  This restatement is pinned against the reference's own
// shader code run on the CPU (oracle/_ref, built by the Makefile from
// shaders/ray_trace.comp.hybrid.hlsl through hlsl2cpp.py) on identical inputs:
// closest hits and rendered frames must agree bit for bit
// (tests/test_oracle_pin.py), and against golden fixtures generated that way
// (tests/golden/).
//
// Templated on the arithmetic type.  float reproduces the reference's order of
// operations with ae_math.h intrinsics (the ones the kernels use); double is
// the FP64 oracle for image error, with libm transcendentals, the same RNG
// stream (each draw widened exactly) and the same estimator.
//
// Every function cites the reference lines it restates.  `hybrid:N` is
// shaders/ray_trace.comp.hybrid.hlsl line N.
#include <omp.h>

#include <cmath>
#include <cstdint>
#include <cstring>

#include "../aviatorengine2_b200/csrc/ae_math.h"
#include "../include/ae_b200.h"

namespace oracle {

// ---------------------------------------------------------------------------
// Arithmetic per type
// ---------------------------------------------------------------------------
template <class T> struct M;
template <> struct M<float> {
    static float sqrt(float x) { return AE_SQRT(x); }
    static float sin(float x) { return ae::sinf_(x); }
    static float cos(float x) { return ae::cosf_(x); }
    static float tan(float x) { return ae::tanf_(x); }
    static float pow(float x, float y) { return ae::powf_(x, y); }
    static float log(float x) { return ae::logf_(x); }
    static float acos(float x) { return ae::acosf_(x); }
    static float atan2(float y, float x) { return ae::atan2f_(y, x); }
    static float fmin(float a, float b) { return AE_FMIN(a, b); }
    static float fmax(float a, float b) { return AE_FMAX(a, b); }
    static float rnd(float u) { return u; }
};
template <> struct M<double> {
    static double sqrt(double x) { return std::sqrt(x); }
    static double sin(double x) { return std::sin(x); }
    static double cos(double x) { return std::cos(x); }
    static double tan(double x) { return std::tan(x); }
    static double pow(double x, double y) {
        // Integer exponents multiply exactly, as the float intrinsic does.
        if (y == std::floor(y) && std::fabs(y) <= 64) {
            int n = int(std::fabs(y));
            double b = x, a = 1;
            while (n) { if (n & 1) a *= b; n >>= 1; if (n) b *= b; }
            return y < 0 ? 1 / a : a;
        }
        return std::pow(x, y);
    }
    static double log(double x) { return std::log(x); }
    static double acos(double x) { return std::acos(x); }
    static double atan2(double y, double x) { return std::atan2(y, x); }
    static double fmin(double a, double b) { return std::fmin(a, b); }
    static double fmax(double a, double b) { return std::fmax(a, b); }
};

template <class T> struct V {
    T x, y, z;
};
template <class T> V<T> v3(T x, T y, T z) { return V<T>{x, y, z}; }
template <class T> V<T> operator+(V<T> a, V<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> V<T> operator-(V<T> a, V<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> V<T> operator*(V<T> a, V<T> b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
template <class T> V<T> operator/(V<T> a, V<T> b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
template <class T> V<T> operator*(V<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> V<T> operator*(T s, V<T> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class T> V<T> operator/(V<T> a, T s) { return {a.x / s, a.y / s, a.z / s}; }
template <class T> V<T> operator/(T s, V<T> a) { return {s / a.x, s / a.y, s / a.z}; }
template <class T> V<T> operator-(V<T> a) { return {-a.x, -a.y, -a.z}; }
template <class T> T dot(V<T> a, V<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> V<T> cross(V<T> a, V<T> b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class T> T len(V<T> a) { return M<T>::sqrt(dot(a, a)); }
template <class T> V<T> nrm(V<T> a) { return a * (T(1) / M<T>::sqrt(dot(a, a))); }
template <class T> V<T> vmin(V<T> a, V<T> b) { return {M<T>::fmin(a.x, b.x), M<T>::fmin(a.y, b.y), M<T>::fmin(a.z, b.z)}; }
template <class T> V<T> vmax(V<T> a, V<T> b) { return {M<T>::fmax(a.x, b.x), M<T>::fmax(a.y, b.y), M<T>::fmax(a.z, b.z)}; }
template <class T> T maxc(V<T> a) { return M<T>::fmax(a.x, M<T>::fmax(a.y, a.z)); }
template <class T> T sat(T x) { return M<T>::fmin(M<T>::fmax(x, T(0)), T(1)); }
template <class T> T sgn(T x) { return x > 0 ? T(1) : (x < 0 ? T(-1) : T(0)); }
template <class T> V<T> reflectv(V<T> i, V<T> n) { return i - (T(2) * dot(n, i)) * n; }
template <class T> V<T> refractv(V<T> i, V<T> n, T eta) {
    const T c = dot(n, i);
    const T k = T(1) - eta * eta * (T(1) - c * c);
    if (k < 0) return v3<T>(0, 0, 0);
    return eta * i - (eta * c + M<T>::sqrt(k)) * n;
}
// rotate(q, v), math/quat.hpp:211-217; hybrid:521-526
template <class T> V<T> qrot(T qx, T qy, T qz, T qw, V<T> v) {
    const V<T> u{qx, qy, qz};
    const V<T> t = T(2) * cross(u, v);
    return v + qw * t + cross(u, t);
}

// The per-invocation RNG (hybrid:238-243).  The draw is computed in float
// and widened exactly for the FP64 oracle, so both consume one stream.
struct Rng {
    uint32_t seed;
    template <class T> T next() { return T(ae::rng_next(seed)); }
};

// Traffic counters: what a ray touches, by the formula of the roofline
// (48 B per node, 128 B per object record, 48 B per instance record, 48 B per
// triangle = 12 B indices + 36 B positions, 60 B for the winner's attributes).
struct Counters {
    uint64_t tlas_nodes = 0, objects = 0, instances = 0, blas_nodes = 0, tris = 0, winners = 0;
    uint64_t bytes() const {
        return 48 * tlas_nodes + 128 * objects + 48 * instances + 48 * blas_nodes + 48 * tris + 60 * winners;
    }
};

struct Scene {
    const ae_object *objects;
    uint32_t n_objects;
    const ae_bvh_node *tlas;
    uint32_t n_nodes;
    const uint32_t *lights;
    uint32_t n_lights;
    const ae_vertex *vertices;
    const uint32_t *indices;
    const ae_bvh_node *blas;
    const ae_instance *instances;
    // material texture array: RGBA8 sRGB words, layer-major (0 layers: none)
    const uint32_t *tex;
    uint32_t tex_w, tex_h, tex_layers;
};

template <class T> struct Ray {
    V<T> o, d;
    T time;
};

template <class T> struct Hit {
    T t = 0;
    V<T> p{0, 0, 0}, n{0, 0, 0};
    T u = 0, v = 0;     // surface uv (interpolated for meshes)
    bool front = true;
    const ae_object *obj = nullptr;
    uint32_t slot = AE_MISS, prim = AE_MISS;
    T alpha = 0, beta = 0;
};

template <class T> V<T> pos(const ae_object &o) { return v3<T>(o.x, o.y, o.z); }
template <class T> V<T> pos2(const ae_object &o) { return v3<T>(o.x2, o.y2, o.z2); }
template <class T> V<T> edge_u(const ae_object &o) { return v3<T>(o.u_x, o.u_y, o.u_z); }
template <class T> V<T> edge_v(const ae_object &o) { return v3<T>(o.v_x, o.v_y, o.v_z); }
template <class T> V<T> albedo(const ae_object &o) { return v3<T>(o.r, o.g, o.b); }

// ---------------------------------------------------------------------------
// Intersection
// ---------------------------------------------------------------------------

// Slab test, hybrid:547-562.
template <class T> bool slab(V<T> o, V<T> inv, const ae_bvh_node &n, T tnear, T tfar) {
    const V<T> t0 = (v3<T>(n.min_x, n.min_y, n.min_z) - o) * inv;
    const V<T> t1 = (v3<T>(n.max_x, n.max_y, n.max_z) - o) * inv;
    const V<T> lo = vmin(t0, t1), hi = vmax(t0, t1);
    const T tmin = M<T>::fmax(M<T>::fmax(lo.x, lo.y), M<T>::fmax(lo.z, tnear));
    const T tmax = M<T>::fmin(M<T>::fmin(hi.x, hi.y), M<T>::fmin(hi.z, tfar));
    return tmin <= tmax;
}

// Sphere span, hybrid:285-297.
template <class T> bool sphere_span(const ae_object &s, const Ray<T> &r, T &t0, T &t1) {
    const V<T> c = pos<T>(s) + r.time * (pos2<T>(s) - pos<T>(s));
    const V<T> oc = c - r.o;
    const T a = dot(r.d, r.d), b = dot(r.d, oc);
    const T cc = dot(oc, oc) - T(s.radius) * T(s.radius);
    const T disc = b * b - a * cc;
    if (disc < 0) { t0 = t1 = 0; return false; }
    const T sq = M<T>::sqrt(disc);
    t0 = (b - sq) / a;
    t1 = (b + sq) / a;
    return true;
}

// Box in its yawed frame, hybrid:315-348.
template <class T> struct BoxLocal {
    V<T> o, d;
    T tin, tout;
    V<T> nin, nout;
};
template <class T> V<T> yaw_rotate(V<T> v, T s, T c) { return v3<T>(c * v.x + s * v.z, v.y, -s * v.x + c * v.z); }
template <class T> bool box_span(const ae_object &b, const Ray<T> &r, BoxLocal<T> &L) {
    const T s = M<T>::sin(T(b.rotation)), c = M<T>::cos(T(b.rotation));
    L.o = yaw_rotate(r.o - pos<T>(b), -s, c);
    L.d = yaw_rotate(r.d, -s, c);
    const V<T> inv = T(1) / L.d;
    const V<T> h = v3<T>(b.half_x, b.half_y, b.half_z);
    const V<T> t0 = (-h - L.o) * inv, t1 = (h - L.o) * inv;
    const V<T> lo = vmin(t0, t1), hi = vmax(t0, t1);
    L.tin = M<T>::fmax(M<T>::fmax(lo.x, lo.y), lo.z);
    L.tout = M<T>::fmin(M<T>::fmin(hi.x, hi.y), hi.z);
    L.nin = v3<T>(0, 0, -sgn(L.d.z));
    if (L.tin == lo.x) L.nin = v3<T>(-sgn(L.d.x), 0, 0);
    else if (L.tin == lo.y) L.nin = v3<T>(0, -sgn(L.d.y), 0);
    L.nout = v3<T>(0, 0, sgn(L.d.z));
    if (L.tout == hi.x) L.nout = v3<T>(sgn(L.d.x), 0, 0);
    else if (L.tout == hi.y) L.nout = v3<T>(0, sgn(L.d.y), 0);
    return L.tout > L.tin;
}

template <class T> void face(Hit<T> &h, V<T> d) {
    h.front = dot(d, h.n) < 0;
    if (!h.front) h.n = -h.n;
}

// get_sphere_uv, hybrid:257-265.
template <class T> void sphere_uv(V<T> p, T rot, T &u, T &v) {
    const T tau = T(6.2831853f), pi = T(3.14159265f);
    const T theta = M<T>::acos(-p.y);
    const T phi = M<T>::atan2(-p.z, p.x) + pi;
    const T x = phi / tau - rot / tau;
    u = x - std::floor(x);
    v = theta / pi;
}

// HitSphere, hybrid:382-423.
template <class T> bool hit_sphere(const ae_object &s, const Ray<T> &r, T tn, T tf, Hit<T> &h) {
    T t0, t1;
    if (!sphere_span(s, r, t0, t1)) return false;
    T root = t0;
    if (root <= tn || tf <= root) {
        root = t1;
        if (root <= tn || tf <= root) return false;
    }
    const V<T> c = pos<T>(s) + r.time * (pos2<T>(s) - pos<T>(s));
    h.t = root;
    h.p = r.o + r.d * root;
    h.n = (h.p - c) / T(s.radius);
    face(h, r.d);
    sphere_uv(h.n, T(s.rotation), h.u, h.v);
    return true;
}

// HitQuad, hybrid:425-478; HitTriangle, hybrid:480-513 (tri = true).
template <class T> bool hit_planar(const ae_object &q, const Ray<T> &r, T tn, T tf, Hit<T> &h, bool tri) {
    const V<T> U = edge_u<T>(q), W = edge_v<T>(q), P = pos<T>(q);
    const V<T> n = cross(U, W);
    const T nn = dot(n, n);
    if (nn < T(1e-8f)) return false;
    const V<T> unit = n / M<T>::sqrt(nn);
    const V<T> w = n / nn;
    T t;
    if (!tri) {
        const T D = dot(n, P);
        const T den = dot(n, r.d);
        if (std::fabs(den) < T(1e-8f)) return false;
        t = (D - dot(n, r.o)) / den;
    } else {
        const T den = dot(n, r.d);
        if (std::fabs(den) < T(1e-8f)) return false;
        t = (dot(n, P) - dot(n, r.o)) / den;
    }
    if (t < tn || t > tf) return false;
    const V<T> X = r.o + r.d * t;
    const V<T> pl = X - P;
    const T a = dot(w, cross(pl, W));
    const T b = dot(w, cross(U, pl));
    if (!tri) {
        if (a < 0 || a > 1 || b < 0 || b > 1) return false;
    } else {
        if (a < 0 || b < 0 || a + b > 1) return false;
    }
    h.u = a; h.v = b; h.alpha = a; h.beta = b;
    h.t = t; h.p = X; h.n = unit;
    face(h, r.d);
    return true;
}

// HitMeshTriangle, hybrid:564-598.
template <class T>
bool hit_mesh_triangle(const Ray<T> &r, T tn, T tf, V<T> p0, V<T> p1, V<T> p2, T &t, T &a, T &b, V<T> &geo) {
    t = 0; a = 0; b = 0; geo = v3<T>(0, 0, 1);
    const V<T> e1 = p1 - p0, e2 = p2 - p0;
    const V<T> n = cross(e1, e2);
    const T nn = dot(n, n);
    if (nn < T(1e-12f)) return false;
    const T den = dot(n, r.d);
    if (std::fabs(den) < T(1e-12f)) return false;
    t = (dot(n, p0) - dot(n, r.o)) / den;
    if (t < tn || t > tf) return false;
    const V<T> w = n / nn;
    const V<T> pl = r.o + r.d * t - p0;
    a = dot(w, cross(pl, e2));
    b = dot(w, cross(e1, pl));
    if (a < 0 || b < 0 || a + b > 1) return false;
    geo = n / M<T>::sqrt(nn);
    return true;
}

template <class T> V<T> vpos(const ae_vertex &v) { return v3<T>(v.px, v.py, v.pz); }

// HitMesh, hybrid:600-707, with ToLocal (hybrid:534-543).  A non-rigid
// instance (scale in pad0, neither 0 nor 1) maps the local ray through 1/s;
// t is unchanged by an affine map applied to origin and direction alike.
template <class T>
bool hit_mesh(const Scene &S, const ae_object &obj, const Ray<T> &r, T tn, T tf, Hit<T> &h, Counters *C) {
    const ae_instance &I = S.instances[obj.instanceIndex];
    if (C) C->instances++;
    const T qx = I.qx, qy = I.qy, qz = I.qz, qw = I.qw;
    Ray<T> L;
    L.o = qrot<T>(-qx, -qy, -qz, qw, r.o - v3<T>(I.px, I.py, I.pz));
    L.d = qrot<T>(-qx, -qy, -qz, qw, r.d);
    L.time = r.time;
    if (I.scale != 0.0f && I.scale != 1.0f) {
        const T inv = T(1) / T(I.scale);
        L.o = L.o * inv;
        L.d = L.d * inv;
    }
    const V<T> invd = T(1) / L.d;
    int stack[64];
    int sp = 0;
    stack[sp++] = 0;
    bool found = false;
    T closest = tf, ba = 0, bb = 0;
    uint32_t best = 0;
    V<T> bgeo = v3<T>(0, 0, 1);
    while (sp > 0) {
        const ae_bvh_node &n = S.blas[I.blasBase + uint32_t(stack[--sp])];
        if (C) C->blas_nodes++;
        if (!slab(L.o, invd, n, tn, closest)) continue;
        if (n.count > 0) {
            for (int i = 0; i < n.count; i++) {
                const uint32_t base = I.indexBase + uint32_t(n.left + i) * 3u;
                if (C) C->tris++;
                const V<T> p0 = vpos<T>(S.vertices[I.vertexBase + S.indices[base]]);
                const V<T> p1 = vpos<T>(S.vertices[I.vertexBase + S.indices[base + 1]]);
                const V<T> p2 = vpos<T>(S.vertices[I.vertexBase + S.indices[base + 2]]);
                T t, a, b;
                V<T> g;
                if (hit_mesh_triangle(L, tn, closest, p0, p1, p2, t, a, b, g)) {
                    closest = t; found = true; ba = a; bb = b; best = base; bgeo = g;
                }
            }
        } else {
            stack[sp++] = n.left;
            stack[sp++] = n.right;
        }
    }
    if (!found) return false;
    if (C) C->winners++;
    const ae_vertex &A = S.vertices[I.vertexBase + S.indices[best]];
    const ae_vertex &B = S.vertices[I.vertexBase + S.indices[best + 1]];
    const ae_vertex &Cv = S.vertices[I.vertexBase + S.indices[best + 2]];
    const T w0 = T(1) - ba - bb;
    const V<T> sh = nrm(w0 * v3<T>(A.nx, A.ny, A.nz) + ba * v3<T>(B.nx, B.ny, B.nz) + bb * v3<T>(Cv.nx, Cv.ny, Cv.nz));
    V<T> geo = bgeo;
    if (dot(geo, sh) < 0) geo = -geo;
    h.t = closest;
    h.p = r.o + r.d * closest;
    h.n = nrm(qrot<T>(qx, qy, qz, qw, sh));
    h.front = dot(r.d, qrot<T>(qx, qy, qz, qw, geo)) < 0;
    if (!h.front) h.n = -h.n;
    h.u = w0 * T(A.u) + ba * T(B.u) + bb * T(Cv.u);
    h.v = w0 * T(A.v) + ba * T(B.v) + bb * T(Cv.v);
    h.prim = (best - I.indexBase) / 3u;
    h.alpha = ba;
    h.beta = bb;
    return true;
}

// BoxFaceUV, hybrid:711-727; HitBox, hybrid:729-773.
template <class T> bool hit_box(const ae_object &b, const Ray<T> &r, T tn, T tf, Hit<T> &h) {
    BoxLocal<T> L;
    if (!box_span(b, r, L)) return false;
    T t = L.tin;
    V<T> ln = L.nin;
    bool outside = true;
    if (t <= tn || tf <= t) {
        t = L.tout; ln = L.nout; outside = false;
        if (t <= tn || tf <= t) return false;
    }
    const T s = M<T>::sin(T(b.rotation)), c = M<T>::cos(T(b.rotation));
    h.t = t;
    h.p = r.o + r.d * t;
    const V<T> lp = L.o + L.d * t;
    const V<T> he = v3<T>(b.half_x, b.half_y, b.half_z);
    T uu, vv;
    if (std::fabs(ln.x) > T(0.5f)) { uu = lp.z / he.z; vv = lp.y / he.y; }
    else if (std::fabs(ln.y) > T(0.5f)) { uu = lp.x / he.x; vv = lp.z / he.z; }
    else { uu = lp.x / he.x; vv = lp.y / he.y; }
    h.u = sat(uu * T(0.5f) + T(0.5f));
    h.v = sat(vv * T(0.5f) + T(0.5f));
    h.n = yaw_rotate(ln, s, c);
    h.front = outside;
    if (!h.front) h.n = -h.n;
    return true;
}

// HitVolume, hybrid:779-822.  Consumes one draw.
template <class T> bool hit_volume(const ae_object &o, const Ray<T> &r, T tn, T tf, Hit<T> &h, Rng &rng) {
    T a = 0, b = 0;
    if (o.shapeType == AE_SHAPE_SPHERE) {
        if (!sphere_span(o, r, a, b)) return false;
    } else if (o.shapeType == AE_SHAPE_BOX) {
        BoxLocal<T> L;
        if (!box_span(o, r, L)) return false;
        a = L.tin; b = L.tout;
    } else {
        return false;
    }
    a = M<T>::fmax(a, tn);
    b = M<T>::fmin(b, tf);
    if (a >= b) return false;
    const T rl = len(r.d);
    const T inside = (b - a) * rl;
    const T d = -M<T>::log(M<T>::fmax(rng.next<T>(), T(1e-8f))) / M<T>::fmax(T(o.density), T(1e-8f));
    if (d > inside) return false;
    h.t = a + d / rl;
    h.p = r.o + r.d * h.t;
    h.n = v3<T>(0, 1, 0);
    h.front = true;
    h.u = h.v = 0;
    return true;
}

// HitObject dispatch, hybrid:827-856.
template <class T>
bool hit_object(const Scene &S, const ae_object &o, const Ray<T> &r, T tn, T tf, Hit<T> &h, Rng &rng, Counters *C) {
    if (o.colorType == AE_MAT_ISOTROPIC) return hit_volume(o, r, tn, tf, h, rng);
    switch (o.shapeType) {
    case AE_SHAPE_SPHERE: return hit_sphere(o, r, tn, tf, h);
    case AE_SHAPE_QUAD: return hit_planar(o, r, tn, tf, h, false);
    case AE_SHAPE_TRIANGLE: return hit_planar(o, r, tn, tf, h, true);
    case AE_SHAPE_MESH: return hit_mesh(S, o, r, tn, tf, h, C);
    default: return hit_box(o, r, tn, tf, h);
    }
}

// Optional record of every closest-hit query (test diagnostics: the rays of
// one pixel's paths, to replay them through the GPU kernels).
struct RayLog {
    ae_ray *rays;
    uint32_t cap, n;
};
thread_local RayLog *g_ray_log = nullptr;

// TraverseBVH, hybrid:862-917: depth-first, interior nodes push left then
// right, far starts at 1e6 and shrinks with each hit; ties go to the later hit.
template <class T> bool traverse(const Scene &S, const Ray<T> &r, T tn, Hit<T> &out, Rng &rng, Counters *C) {
    if (g_ray_log && g_ray_log->n < g_ray_log->cap) {
        ae_ray &q = g_ray_log->rays[g_ray_log->n++];
        q.ox = float(r.o.x); q.oy = float(r.o.y); q.oz = float(r.o.z); q.tnear = float(tn);
        q.dx = float(r.d.x); q.dy = float(r.d.y); q.dz = float(r.d.z); q.time = float(r.time);
    }
    if (S.n_nodes == 0) return false;
    const V<T> inv = T(1) / r.d;
    int stack[64];
    int sp = 0;
    stack[sp++] = 0;
    bool found = false;
    T tf = T(1000000.0f);
    while (sp > 0) {
        const int ni = stack[--sp];
        const ae_bvh_node &n = S.tlas[ni];
        if (C) C->tlas_nodes++;
        if (!slab(r.o, inv, n, tn, tf)) continue;
        if (n.count > 0) {
            for (int i = 0; i < n.count; i++) {
                const uint32_t slot = uint32_t(n.left + i);
                const ae_object &o = S.objects[slot];
                if (C) C->objects++;
                Hit<T> h;
                if (hit_object(S, o, r, tn, tf, h, rng, C)) {
                    tf = h.t;
                    h.obj = &o;
                    h.slot = slot;
                    out = h;
                    found = true;
                }
            }
        } else {
            stack[sp++] = n.left;
            stack[sp++] = n.right;
        }
    }
    return found;
}

// ---------------------------------------------------------------------------
// Shading
// ---------------------------------------------------------------------------

// textureColor, hybrid:919-925: SampleLevel(uv, layer, 0) with the
// renderer's linear REPEAT sampler on the RGBA8 sRGB array (decode, then
// bilinear).  Float: the shared definition in ae_math.h.  Double: the same
// steps in double (sRGB decode with libm pow).
inline const float *srgb_table() {
    static float lut[256];
    static bool ready = false;
    if (!ready) {
        for (uint32_t b = 0; b < 256; b++) lut[b] = ae::srgb_to_linear(b);
        ready = true;
    }
    return lut;
}
inline V<float> texture_color(const Scene &S, uint32_t layer, float u, float v) {
    const ae::f3 c = ae::texture_sample(S.tex, srgb_table(), S.tex_w, S.tex_h, S.tex_layers, layer, u, v);
    return v3<float>(c.x, c.y, c.z);
}
inline V<double> texture_color(const Scene &S, uint32_t layer, double u, double v) {
    if (S.tex_layers == 0 || S.tex_w == 0 || S.tex_h == 0) return v3<double>(1, 1, 1);
    if (layer >= S.tex_layers) layer = S.tex_layers - 1;
    if (!(std::fabs(u) <= 1.7e308)) u = 0;
    if (!(std::fabs(v) <= 1.7e308)) v = 0;
    auto dec = [](uint32_t b) {
        const double c = double(b) / 255.0;
        return c <= 0.04045 ? c / 12.92 : std::pow((c + 0.055) / 1.055, 2.4);
    };
    auto wrap = [](double f, uint32_t n) {
        const double g = std::fmin(std::fmax(f, -1073741824.0), 1073741824.0);
        int64_t m = int64_t(g) % int64_t(n);
        return uint32_t(m < 0 ? m + int64_t(n) : m);
    };
    const double x = u * S.tex_w - 0.5, y = v * S.tex_h - 0.5;
    const double fx = std::floor(x), fy = std::floor(y), ax = x - fx, ay = y - fy;
    const uint32_t x0 = wrap(fx, S.tex_w), x1 = wrap(fx + 1, S.tex_w), y0 = wrap(fy, S.tex_h), y1 = wrap(fy + 1, S.tex_h);
    const uint32_t *L = S.tex + size_t(layer) * S.tex_w * S.tex_h;
    auto tx = [&](uint32_t xx, uint32_t yy) {
        const uint32_t t = L[size_t(yy) * S.tex_w + xx];
        return v3<double>(dec(t & 0xff), dec((t >> 8) & 0xff), dec((t >> 16) & 0xff));
    };
    const V<double> top = tx(x0, y0) + (tx(x1, y0) - tx(x0, y0)) * ax;
    const V<double> bot = tx(x0, y1) + (tx(x1, y1) - tx(x0, y1)) * ax;
    return top + (bot - top) * ay;
}

// SurfaceAlbedo, hybrid:940-949: the flat albedo, or the texel at the hit's
// UV tinted by it (texel * lerp(1, albedo, TextureTint)).
template <class T> V<T> surface_albedo(const Scene &S, const Hit<T> &h) {
    if (h.obj->textureID == AE_NO_TEXTURE) return albedo<T>(*h.obj);
    const V<T> texel = texture_color(S, h.obj->textureID, h.u, h.v);
    const V<T> one = v3<T>(1, 1, 1);
    return texel * (one + T(h.obj->textureTint) * (albedo<T>(*h.obj) - one));
}

template <class T> V<T> random_direction(Rng &rng) {
    // hybrid:245-251
    const T z = rng.next<T>() * T(2) - T(1);
    const T a = rng.next<T>() * T(6.2831853f);
    const T rr = M<T>::sqrt(T(1) - z * z);
    return v3<T>(rr * M<T>::cos(a), rr * M<T>::sin(a), z);
}

// GGX metal, the library's extension of the materials (not a reference
// material): Walter, Marschner, Li and Torrance, "Microfacet Models for
// Refraction through Rough Surfaces" (EGSR 2007), alpha = roughness (fuzz).
// The half vector m is drawn with density D(m)|m.n| (eqs. 35-36), the
// direction is the mirror of i = -d about m (eq. 39), and the sample weight
// is F(i.m) |i.m| G(i,o,m) / (|i.n| |m.n|) (eq. 41) with Smith's
// G1(v) = 2 / (1 + sqrt(1 + alpha^2 tan^2 theta_v)) (eq. 34) and Schlick's
// Fresnel with F0 = albedo.  The tangent frame around n is Duff et al.'s
// (JCGT 2017).  Two RNG draws, always taken.
template <class T> T ggx_g1(T cv, T a2) {
    const T c2 = cv * cv;
    const T t2 = (T(1) - c2) / c2;
    return T(2) / (T(1) + M<T>::sqrt(T(1) + a2 * t2));
}
template <class T>
bool ggx_bounce(V<T> d, V<T> n, V<T> alb, T alpha, V<T> &dir, V<T> &weight, Rng &rng) {
    const V<T> i = -nrm(d);
    const T u1 = rng.next<T>();
    const T u2 = rng.next<T>();
    const T cin = dot(i, n);
    if (cin <= 0) return false;
    const T a2 = alpha * alpha;
    const T c2 = (T(1) - u1) / (T(1) + (a2 - T(1)) * u1);
    const T cm = M<T>::sqrt(c2);
    const T sm = M<T>::sqrt(M<T>::fmax(T(0), T(1) - c2));
    const T phi = T(6.2831853f) * u2;
    const T cp = M<T>::cos(phi), sp = M<T>::sin(phi);
    const T sg = n.z >= 0 ? T(1) : T(-1);
    const T a = T(-1) / (sg + n.z);
    const T b = (n.x * n.y) * a;
    const V<T> t = v3<T>(T(1) + (sg * (n.x * n.x)) * a, sg * b, -(sg * n.x));
    const V<T> bt = v3<T>(b, sg + (n.y * n.y) * a, -n.y);
    const V<T> m = t * (sm * cp) + bt * (sm * sp) + n * cm;
    const T im = dot(i, m);
    if (im <= 0) return false;
    dir = m * (T(2) * im) - i;
    const T con = dot(dir, n);
    if (con <= 0) return false;
    const T g = ggx_g1(cin, a2) * ggx_g1(con, a2);
    const T w = (im * g) / (cin * cm);
    const T f5 = M<T>::pow(T(1) - im, T(5));
    const V<T> fr = alb + (v3<T>(1, 1, 1) - alb) * f5;
    weight = fr * w;
    return true;
}

// GetBounce, hybrid:965-1033.
template <class T> bool bounce(const Ray<T> &r, const Hit<T> &h, V<T> &dir, Rng &rng) {
    dir = v3<T>(0, 0, 0);
    switch (h.obj->colorType) {
    case AE_MAT_LAMBERTIAN:
        dir = h.n + random_direction<T>(rng);
        if (dot(dir, dir) < T(0.001f)) dir = h.n;
        return true;
    case AE_MAT_METAL: {
        dir = nrm(reflectv(r.d, h.n));
        dir = dir + random_direction<T>(rng) * T(h.obj->fuzz);
        return dot(dir, h.n) > 0;
    }
    case AE_MAT_DIELECTRIC: {
        const T ior = h.obj->refraction;
        const T ri = h.front ? T(1) / ior : ior;
        const V<T> d = nrm(r.d);
        const T ct = M<T>::fmin(dot(-d, h.n), T(1));
        const T st = M<T>::sqrt(M<T>::fmax(T(0), T(1) - ct * ct));
        const T r0 = M<T>::pow((T(1) - ri) / (T(1) + ri), T(2));
        const T refl = r0 + (T(1) - r0) * M<T>::pow(T(1) - ct, T(5));
        if (ri * st > T(1) || refl > rng.next<T>()) dir = reflectv(d, h.n);
        else dir = refractv(d, h.n, ri);
        return true;
    }
    case AE_MAT_ISOTROPIC:
        dir = random_direction<T>(rng);
        return true;
    default:
        return false;
    }
}

// SampleLight, hybrid:1057-1119.
template <class T> void sample_light(const ae_object &L, V<T> from, V<T> &p, T &omega, Rng &rng) {
    p = pos<T>(L);
    omega = 0;
    if (L.shapeType == AE_SHAPE_QUAD) {
        const T r1 = rng.next<T>();
        const T r2 = rng.next<T>();
        p = pos<T>(L) + r1 * edge_u<T>(L) + r2 * edge_v<T>(L);
        const V<T> cuv = cross(edge_u<T>(L), edge_v<T>(L));
        const T area = len(cuv);
        const V<T> ln = cuv / M<T>::fmax(area, T(1e-8f));
        V<T> ts = from - p;
        const T d2 = dot(ts, ts);
        ts = nrm(ts);
        const T cl = std::fabs(dot(ln, ts));
        omega = (cl * area) / M<T>::fmax(d2, T(1e-8f));
        return;
    }
    if (L.shapeType == AE_SHAPE_SPHERE) {
        const V<T> tl = pos<T>(L) - from;
        const T d2 = M<T>::fmax(dot(tl, tl), T(1e-8f));
        const T r2 = T(L.radius) * T(L.radius);
        p = pos<T>(L);
        if (d2 <= r2) { omega = T(4) * T(3.14159265f); return; }
        const T ctm = M<T>::sqrt(M<T>::fmax(T(0), T(1) - r2 / d2));
        omega = T(2) * T(3.14159265f) * (T(1) - ctm);
        return;
    }
    const V<T> tl = pos<T>(L) - from;
    const T d2 = M<T>::fmax(dot(tl, tl), T(1e-8f));
    const T area = T(4) * (T(L.half_x) * T(L.half_y) + T(L.half_y) * T(L.half_z) + T(L.half_z) * T(L.half_x)) / T(6);
    omega = area / d2;
}

// CalculateDirectLight, hybrid:1122-1212: every light, one sample each; the
// shadow ray steps through up to four dielectric hits.
template <class T> V<T> direct_light(const Scene &S, const Hit<T> &h, const Ray<T> &r, Rng &rng, Counters *C) {
    V<T> acc = v3<T>(0, 0, 0);
    for (uint32_t i = 0; i < S.n_lights; i++) {
        const ae_object &L = S.objects[S.lights[i]];
        V<T> lp;
        T omega;
        sample_light(L, h.p, lp, omega, rng);
        if (omega <= 0) continue;
        V<T> sd = lp - h.p;
        const T dist = len(sd);
        if (dist <= T(1e-6f)) continue;
        sd = sd / dist;
        const T ct = dot(h.n, sd);
        if (ct <= 0) continue;
        Ray<T> sr;
        sr.o = h.p + h.n * T(0.001f);
        sr.d = sd;
        sr.time = r.time;
        bool occluded = false;
        for (int k = 0; k < 4; k++) {
            Hit<T> sh;
            if (!traverse(S, sr, T(0.001f), sh, rng, C)) break;
            if (sh.t >= len(lp - sr.o) - T(0.001f)) break;
            if (sh.obj->colorType == AE_MAT_DIFFUSE_LIGHT) break;
            if (sh.obj->colorType != AE_MAT_DIELECTRIC) { occluded = true; break; }
            sr.o = sh.p + sr.d * T(0.001f);
        }
        if (!occluded) {
            const V<T> rad = T(L.emission) * albedo<T>(L);
            const V<T> brdf = surface_albedo(S, h);
            acc = acc + brdf * rad * ct * omega;
        }
    }
    return acc;
}

// ColorRay, hybrid:1230-1325.
template <class T> V<T> color_ray(const Scene &S, const ae_config &cfg, Ray<T> ray, Rng &rng, Counters *C) {
    V<T> thr = v3<T>(1, 1, 1), acc = v3<T>(0, 0, 0);
    const V<T> sky = v3<T>(cfg.sky_r, cfg.sky_g, cfg.sky_b);
    for (uint32_t b = 0; b < cfg.depth; b++) {
        Hit<T> h;
        if (!traverse(S, ray, T(0.001f), h, rng, C)) {
            acc = acc + thr * sky;
            break;
        }
        if (h.obj->colorType == AE_MAT_DIFFUSE_LIGHT) {
            acc = acc + thr * (T(h.obj->emission) * albedo<T>(*h.obj));
            break;
        }
        if (h.obj->colorType == AE_MAT_LAMBERTIAN) {
            V<T> dl = direct_light(S, h, ray, rng, C);
            const T luma = maxc(dl);
            if (luma > T(8)) dl = dl * (T(8) / luma);
            acc = acc + thr * dl;
        }
        V<T> sd, gw;
        const bool ggx = h.obj->colorType == AE_MAT_GGX_METAL;
        if (ggx ? !ggx_bounce(ray.d, h.n, surface_albedo(S, h), T(h.obj->fuzz), sd, gw, rng)
                : !bounce(ray, h, sd, rng))
            break;
        ray.d = nrm(sd);
        const T sign = dot(ray.d, h.n) < 0 ? T(-1) : T(1);
        ray.o = h.p + h.n * (T(0.001f) * sign);
        if (ggx) thr = thr * gw;
        else if (h.obj->colorType != AE_MAT_DIELECTRIC) thr = thr * surface_albedo(S, h);
        if (b > 0) {
            T p = maxc(thr);
            p = M<T>::fmin(M<T>::fmax(p, T(0.1f)), T(1));
            if (rng.next<T>() > p) break;
            thr = thr / p;
        }
    }
    return acc;
}

// Camera basis of main, hybrid:1347-1361.
template <class T> struct Camera {
    V<T> src, u, v, pu, pv, p0, du, dv;
    T defocus;
};
template <class T> Camera<T> camera(const ae_config &c) {
    Camera<T> K;
    K.src = v3<T>(c.source_x, c.source_y, c.source_z);
    const V<T> tgt = v3<T>(c.target_x, c.target_y, c.target_z), up = v3<T>(c.up_x, c.up_y, c.up_z);
    const V<T> w = nrm(K.src - tgt);
    K.u = nrm(cross(up, w));
    K.v = cross(w, K.u);
    const T deg = T(0.017453292519943295f);
    const T vh = T(2) * M<T>::tan((T(c.fov) / T(2)) * deg) * T(c.focus_dist);
    const T vw = vh * T(c.width) / T(c.height);
    const V<T> vu = vw * K.u, vv = vh * -K.v;
    K.pu = vu / T(c.width);
    K.pv = vv / T(c.height);
    K.p0 = K.src - T(c.focus_dist) * w - vu / T(2) - vv / T(2) + K.pu / T(2) + K.pv / T(2);
    const T dr = T(c.focus_dist) * M<T>::tan((T(c.defocus_angle) / T(2)) * deg);
    K.du = K.u * dr;
    K.dv = K.v * dr;
    K.defocus = c.defocus_angle;
    return K;
}

// One pixel's frame radiance (main, hybrid:1346-1386), before blending.
template <class T> V<T> pixel_radiance(const Scene &S, const ae_config &c, const Camera<T> &K, uint32_t x, uint32_t y, Counters *C) {
    Rng rng{x + y * c.width + c.batch * c.width * c.height + 1u};
    V<T> color = v3<T>(0, 0, 0);
    const uint32_t spp = c.batches ? (c.samples / c.batches > 1u ? c.samples / c.batches : 1u) : 1u;
    for (uint32_t s = 0; s < spp; s++) {
        const T jx = rng.next<T>() - T(0.5f);
        const T jy = rng.next<T>() - T(0.5f);
        const V<T> tgt = K.p0 + (T(x) + jx) * K.pu + (T(y) + jy) * K.pv;
        Ray<T> r;
        if (K.defocus <= 0) {
            r.o = K.src;
        } else {
            T px, py;
            for (;;) {  // random_in_unit_disk, hybrid:1215-1221
                const T a = rng.next<T>(), b = rng.next<T>();
                px = a * T(2) - T(1);
                py = b * T(2) - T(1);
                if (M<T>::sqrt(px * px + py * py + T(0) * T(0)) < T(1)) break;
            }
            r.o = K.src + px * K.du + py * K.dv;
        }
        r.d = nrm(tgt - r.o);
        r.time = rng.next<T>();
        color = color + color_ray(S, c, r, rng, C);
    }
    return color / T(spp);
}

// ToneMapACES and LinearToSRGB, hybrid:213-233.
template <class T> V<T> aces(V<T> x) {
    const T a = T(2.51f), b = T(0.03f), c = T(2.43f), d = T(0.59f), e = T(0.14f);
    const V<T> n = x * (a * x + v3<T>(b, b, b));
    const V<T> m = x * (c * x + v3<T>(d, d, d)) + v3<T>(e, e, e);
    const V<T> q = n / m;
    return v3<T>(sat(q.x), sat(q.y), sat(q.z));
}
template <class T> T srgb1(T c) {
    const T lo = c * T(12.92f);
    const T hi = T(1.055f) * M<T>::pow(c, T(1.0f) / T(2.4f)) - T(0.055f);
    return c <= T(0.0031308f) ? lo : hi;
}
template <class T> V<T> srgb(V<T> c) {
    c = v3<T>(sat(c.x), sat(c.y), sat(c.z));
    return v3<T>(srgb1(c.x), srgb1(c.y), srgb1(c.z));
}

template <class T>
void render_frame(const Scene &S, const ae_config &c, T *accum, T *display, T *frame, const uint32_t *xy, uint32_t n_px,
                  int threads) {
    if (threads > 0) omp_set_num_threads(threads);
    const Camera<T> K = camera<T>(c);
    const int64_t total = xy ? int64_t(n_px) : int64_t(c.width) * c.height;
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < total; i++) {
        uint32_t x, y;
        if (xy) { x = xy[2 * i]; y = xy[2 * i + 1]; }
        else { x = uint32_t(i % c.width); y = uint32_t(i / c.width); }
        const size_t px = size_t(y) * c.width + x;
        T *acc = accum + 4 * px;
        if (c.displayOnly) {
            const V<T> g = srgb(aces(v3<T>(acc[0], acc[1], acc[2]) * T(c.exposure)));
            T *d = display + 4 * px;
            d[0] = g.x; d[1] = g.y; d[2] = g.z; d[3] = 1;
            continue;
        }
        const V<T> col = pixel_radiance<T>(S, c, K, x, y, nullptr);
        if (frame) { T *f = frame + 4 * px; f[0] = col.x; f[1] = col.y; f[2] = col.z; f[3] = 1; }
        V<T> a;
        if (c.batch == 0) a = col;
        else {
            const T w = T(1) / T(c.batch + 1);
            const V<T> prev = v3<T>(acc[0], acc[1], acc[2]);
            a = prev + w * (col - prev);
        }
        acc[0] = a.x; acc[1] = a.y; acc[2] = a.z; acc[3] = 1;
        const V<T> g = srgb(aces(a * T(c.exposure)));
        T *d = display + 4 * px;
        d[0] = g.x; d[1] = g.y; d[2] = g.z; d[3] = 1;
    }
}

}  // namespace oracle

using namespace oracle;

extern "C" {

// ae_hit per ray; counters (optional) receive 6 aggregates:
// tlas_nodes, objects, instances, blas_nodes, tris, winners.
int oracle_closest_hit(const Scene *S, const ae_ray *rays, uint32_t n, ae_hit *hits, uint64_t *counters, int threads) {
    if (threads > 0) omp_set_num_threads(threads);
    uint64_t agg[6] = {0, 0, 0, 0, 0, 0};
#pragma omp parallel
    {
        Counters C;
#pragma omp for schedule(dynamic, 1024)
        for (int64_t i = 0; i < int64_t(n); i++) {
            const ae_ray &q = rays[i];
            Ray<float> r;
            r.o = v3<float>(q.ox, q.oy, q.oz);
            r.d = v3<float>(q.dx, q.dy, q.dz);
            r.time = q.time;
            Rng rng{1u};
            Hit<float> h;
            ae_hit out{0, 0, 0, AE_MISS, AE_MISS};
            if (traverse(*S, r, q.tnear, h, rng, counters ? &C : nullptr)) {
                out.t = h.t;
                out.alpha = h.alpha;
                out.beta = h.beta;
                out.object = h.slot;
                out.prim = h.prim;
            }
            hits[i] = out;
        }
        if (counters) {
#pragma omp critical
            {
                agg[0] += C.tlas_nodes; agg[1] += C.objects; agg[2] += C.instances;
                agg[3] += C.blas_nodes; agg[4] += C.tris; agg[5] += C.winners;
            }
        }
    }
    if (counters) std::memcpy(counters, agg, sizeof(agg));
    return 0;
}

// Frame render in float (parity) or double (image-error oracle).  Buffers are
// width*height*4 of the precision's type.  xy (optional) restricts the frame
// to n_px listed pixels.
int oracle_render_frame_f32(const Scene *S, const ae_config *c, float *accum, float *display, float *frame,
                            const uint32_t *xy, uint32_t n_px, int threads) {
    render_frame<float>(*S, *c, accum, display, frame, xy, n_px, threads);
    return 0;
}
int oracle_render_frame_f64(const Scene *S, const ae_config *c, double *accum, double *display, double *frame,
                            const uint32_t *xy, uint32_t n_px, int threads) {
    render_frame<double>(*S, *c, accum, display, frame, xy, n_px, threads);
    return 0;
}

// Every closest-hit query of pixel (x, y)'s samples in one float frame, in
// order (camera, shadow and bounce rays); returns how many were made.
uint32_t oracle_pixel_rays(const Scene *S, const ae_config *c, uint32_t x, uint32_t y, ae_ray *out, uint32_t cap) {
    RayLog log{out, cap, 0};
    g_ray_log = &log;
    const Camera<float> K = camera<float>(*c);
    pixel_radiance<float>(*S, *c, K, x, y, nullptr);
    g_ray_log = nullptr;
    return log.n;
}

// The shared intrinsics on the host, for their accuracy tests:
// fn 0 sin, 1 cos, 2 tan, 3 exp, 4 log, 5 pow(x, y), 6 atan2(x, y), 7 acos, 8 rng draw of seed x.
int oracle_math(int fn, const float *x, const float *y, float *out, uint32_t n) {
    for (uint32_t i = 0; i < n; i++) {
        switch (fn) {
        case 0: out[i] = ae::sinf_(x[i]); break;
        case 1: out[i] = ae::cosf_(x[i]); break;
        case 2: out[i] = ae::tanf_(x[i]); break;
        case 3: out[i] = ae::expf_(x[i]); break;
        case 4: out[i] = ae::logf_(x[i]); break;
        case 5: out[i] = ae::powf_(x[i], y[i]); break;
        case 6: out[i] = ae::atan2f_(x[i], y[i]); break;
        case 7: out[i] = ae::acosf_(x[i]); break;
        default: { uint32_t sd; std::memcpy(&sd, &x[i], 4); out[i] = ae::rng_next(sd); }
        }
    }
    return 0;
}

// `count` GGX metal samples in double (ggx_bounce above) for incoming
// direction d, shading normal n, albedo alb and roughness alpha, RNG seeds
// seed, seed + 1, ...: out[7 k ..] = direction xyz, weight xyz, 1 if the path
// continues (else 0 and the rest zero).
int oracle_ggx_samples(const double *d, const double *n, const double *alb, double alpha, uint32_t seed,
                       uint32_t count, double *out) {
    for (uint32_t k = 0; k < count; k++) {
        Rng rng{seed + k};
        V<double> dir = v3<double>(0, 0, 0), w = v3<double>(0, 0, 0);
        const bool ok = ggx_bounce<double>(v3<double>(d[0], d[1], d[2]), v3<double>(n[0], n[1], n[2]),
                                           v3<double>(alb[0], alb[1], alb[2]), alpha, dir, w, rng);
        double *o = out + 7 * size_t(k);
        o[0] = ok ? dir.x : 0; o[1] = ok ? dir.y : 0; o[2] = ok ? dir.z : 0;
        o[3] = ok ? w.x : 0; o[4] = ok ? w.y : 0; o[5] = ok ? w.z : 0;
        o[6] = ok ? 1 : 0;
    }
    return 0;
}

// Camera rays of a frame (main, hybrid:1346-1373), row-major.
int oracle_camera_rays(const ae_config *c, ae_ray *out) {
    const Camera<float> K = camera<float>(*c);
    for (uint32_t y = 0; y < c->height; y++)
        for (uint32_t x = 0; x < c->width; x++) {
            Rng rng{x + y * c->width + c->batch * c->width * c->height + 1u};
            const float jx = rng.next<float>() - 0.5f;
            const float jy = rng.next<float>() - 0.5f;
            const V<float> tgt = K.p0 + (float(x) + jx) * K.pu + (float(y) + jy) * K.pv;
            V<float> o = K.src;
            if (K.defocus > 0) {
                float px, py;
                for (;;) {
                    const float a = rng.next<float>(), b = rng.next<float>();
                    px = a * 2.0f - 1.0f;
                    py = b * 2.0f - 1.0f;
                    if (M<float>::sqrt(px * px + py * py + 0.0f * 0.0f) < 1.0f) break;
                }
                o = K.src + px * K.du + py * K.dv;
            }
            const V<float> d = nrm(tgt - o);
            ae_ray &r = out[size_t(y) * c->width + x];
            r.ox = o.x; r.oy = o.y; r.oz = o.z; r.tnear = 0.001f;
            r.dx = d.x; r.dy = d.y; r.dz = d.z; r.time = rng.next<float>();
        }
    return 0;
}

// One diffuse bounce per hit, as the library's ray-set generator defines it:
// the pixel's RNG stream after its camera ray, direction n + RandomDirection()
// (hybrid:980-986), origin offset 0.001 along the facing shading normal
// (hybrid:1294-1296); the normal recomputed as HitMesh finishes
// (hybrid:655-706).  valid[i] = 0 where the primary missed or hit a
// non-planar analytic object.
int oracle_bounce_rays(const Scene *S, const ae_config *c, const ae_ray *prim, const ae_hit *hits, uint32_t n,
                       ae_ray *out, uint8_t *valid) {
    const Camera<float> K = camera<float>(*c);
    for (uint32_t i = 0; i < n; i++) {
        out[i] = prim[i];
        valid[i] = 0;
        const ae_hit &h = hits[i];
        if (h.object == AE_MISS) continue;
        const ae_object &obj = S->objects[h.object];
        const V<float> d = v3<float>(prim[i].dx, prim[i].dy, prim[i].dz);
        V<float> sn;
        if (obj.shapeType == AE_SHAPE_MESH) {
            const ae_instance &I = S->instances[obj.instanceIndex];
            const uint32_t base = I.indexBase + h.prim * 3u;
            const ae_vertex &A = S->vertices[I.vertexBase + S->indices[base]];
            const ae_vertex &B = S->vertices[I.vertexBase + S->indices[base + 1]];
            const ae_vertex &C = S->vertices[I.vertexBase + S->indices[base + 2]];
            const float w0 = 1.0f - h.alpha - h.beta;
            const V<float> sh = nrm(w0 * v3<float>(A.nx, A.ny, A.nz) + h.alpha * v3<float>(B.nx, B.ny, B.nz) +
                                    h.beta * v3<float>(C.nx, C.ny, C.nz));
            const V<float> p0 = vpos<float>(A);
            const V<float> gn = cross(vpos<float>(B) - p0, vpos<float>(C) - p0);
            V<float> geo = gn / M<float>::sqrt(dot(gn, gn));
            if (dot(geo, sh) < 0) geo = -geo;
            sn = nrm(qrot<float>(I.qx, I.qy, I.qz, I.qw, sh));
            if (!(dot(d, qrot<float>(I.qx, I.qy, I.qz, I.qw, geo)) < 0)) sn = -sn;
        } else if (obj.shapeType == AE_SHAPE_QUAD || obj.shapeType == AE_SHAPE_TRIANGLE) {
            const V<float> nn = cross(edge_u<float>(obj), edge_v<float>(obj));
            sn = nn / M<float>::sqrt(dot(nn, nn));
            if (!(dot(d, sn) < 0)) sn = -sn;
        } else {
            continue;
        }
        const uint32_t x = i % c->width, y = i / c->width;
        Rng rng{x + y * c->width + c->batch * c->width * c->height + 1u};
        rng.next<float>();
        rng.next<float>();
        if (K.defocus > 0) {
            for (;;) {
                const float a = rng.next<float>(), b = rng.next<float>();
                const float px = a * 2.0f - 1.0f, py = b * 2.0f - 1.0f;
                if (M<float>::sqrt(px * px + py * py + 0.0f * 0.0f) < 1.0f) break;
            }
        }
        rng.next<float>();
        V<float> dir = sn + random_direction<float>(rng);
        if (dot(dir, dir) < 0.001f) dir = sn;
        dir = nrm(dir);
        const V<float> o = v3<float>(prim[i].ox, prim[i].oy, prim[i].oz);
        const V<float> p = o + d * h.t;
        const float sgn = dot(dir, sn) < 0 ? -1.0f : 1.0f;
        const V<float> no = p + sn * (0.001f * sgn);
        ae_ray &r = out[i];
        r.ox = no.x; r.oy = no.y; r.oz = no.z; r.tnear = 0.001f;
        r.dx = dir.x; r.dy = dir.y; r.dz = dir.z;
        valid[i] = 1;
    }
    return 0;
}

// Per-path traffic of one frame's paths (camera, bounce and shadow rays),
// for the Mpaths/s roofline: counters as oracle_closest_hit.
int oracle_path_counters(const Scene *S, const ae_config *c, const uint32_t *xy, uint32_t n_px, uint64_t *counters,
                         uint64_t *rays_traced, int threads) {
    if (threads > 0) omp_set_num_threads(threads);
    const Camera<float> K = camera<float>(*c);
    uint64_t agg[6] = {0, 0, 0, 0, 0, 0};
#pragma omp parallel
    {
        Counters C;
#pragma omp for schedule(dynamic, 64)
        for (int64_t i = 0; i < int64_t(n_px); i++) pixel_radiance<float>(*S, *c, K, xy[2 * i], xy[2 * i + 1], &C);
#pragma omp critical
        {
            agg[0] += C.tlas_nodes; agg[1] += C.objects; agg[2] += C.instances;
            agg[3] += C.blas_nodes; agg[4] += C.tris; agg[5] += C.winners;
        }
    }
    std::memcpy(counters, agg, sizeof(agg));
    if (rays_traced) *rays_traced = 0;
    return 0;
}

}  // extern "C"

// ===========================================================================
// Hybrid renderer passes (float only): deferred resolve, temporal upsample,
// and the library's ray-cast G-buffer.  `deferred:N` is
// shaders/deferred.comp.hlsl line N, `upsample:N` shaders/upsample.comp.hlsl.
// ===========================================================================
namespace oracle {

using Vf = V<float>;

// AABBEntry, deferred:635-646.
inline float aabb_entry(Vf o, Vf inv, const ae_bvh_node &n, float tn, float tf) {
    const Vf t0 = (v3<float>(n.min_x, n.min_y, n.min_z) - o) * inv;
    const Vf t1 = (v3<float>(n.max_x, n.max_y, n.max_z) - o) * inv;
    const Vf lo = vmin(t0, t1), hi = vmax(t0, t1);
    const float tmin = M<float>::fmax(M<float>::fmax(lo.x, lo.y), M<float>::fmax(lo.z, tn));
    const float tmax = M<float>::fmin(M<float>::fmin(hi.x, hi.y), M<float>::fmin(hi.z, tf));
    return tmin <= tmax ? tmin : 1e30f;
}

inline void to_local(const ae_instance &I, const Ray<float> &r, Ray<float> &L) {
    L.o = qrot<float>(-I.qx, -I.qy, -I.qz, I.qw, r.o - v3<float>(I.px, I.py, I.pz));
    L.d = qrot<float>(-I.qx, -I.qy, -I.qz, I.qw, r.d);
    L.time = r.time;
    if (I.scale != 0.0f && I.scale != 1.0f) {
        const float inv = 1.0f / I.scale;
        L.o = L.o * inv;
        L.d = L.d * inv;
    }
}

// HitMesh with nearest-first children, deferred:684-806.
inline bool hit_mesh_ordered(const Scene &S, const ae_object &obj, const Ray<float> &r, float tn, float tf,
                             Hit<float> &h) {
    const ae_instance &I = S.instances[obj.instanceIndex];
    Ray<float> L;
    to_local(I, r, L);
    const Vf invd = 1.0f / L.d;
    int stack[64];
    int sp = 0;
    stack[sp++] = 0;
    bool found = false;
    float closest = tf, ba = 0, bb = 0;
    uint32_t best = 0;
    Vf bgeo = v3<float>(0, 0, 1);
    while (sp > 0) {
        const ae_bvh_node &n = S.blas[I.blasBase + uint32_t(stack[--sp])];
        if (!slab(L.o, invd, n, tn, closest)) continue;
        if (n.count > 0) {
            for (int i = 0; i < n.count; i++) {
                const uint32_t base = I.indexBase + uint32_t(n.left + i) * 3u;
                const Vf p0 = vpos<float>(S.vertices[I.vertexBase + S.indices[base]]);
                const Vf p1 = vpos<float>(S.vertices[I.vertexBase + S.indices[base + 1]]);
                const Vf p2 = vpos<float>(S.vertices[I.vertexBase + S.indices[base + 2]]);
                float t, a, b;
                Vf g;
                if (hit_mesh_triangle(L, tn, closest, p0, p1, p2, t, a, b, g)) {
                    closest = t; found = true; ba = a; bb = b; best = base; bgeo = g;
                }
            }
        } else {
            const ae_bvh_node &Ln = S.blas[I.blasBase + uint32_t(n.left)];
            const ae_bvh_node &Rn = S.blas[I.blasBase + uint32_t(n.right)];
            const float tl = aabb_entry(L.o, invd, Ln, tn, closest);
            const float tr = aabb_entry(L.o, invd, Rn, tn, closest);
            const bool lf = tl <= tr;
            if (M<float>::fmax(tl, tr) < 1e30f) stack[sp++] = lf ? n.right : n.left;
            if (M<float>::fmin(tl, tr) < 1e30f) stack[sp++] = lf ? n.left : n.right;
        }
    }
    if (!found) return false;
    const ae_vertex &A = S.vertices[I.vertexBase + S.indices[best]];
    const ae_vertex &B = S.vertices[I.vertexBase + S.indices[best + 1]];
    const ae_vertex &C = S.vertices[I.vertexBase + S.indices[best + 2]];
    const float w0 = 1.0f - ba - bb;
    const Vf sh = nrm(w0 * v3<float>(A.nx, A.ny, A.nz) + ba * v3<float>(B.nx, B.ny, B.nz) + bb * v3<float>(C.nx, C.ny, C.nz));
    Vf geo = bgeo;
    if (dot(geo, sh) < 0) geo = -geo;
    h.t = closest;
    h.p = r.o + r.d * closest;
    h.n = nrm(qrot<float>(I.qx, I.qy, I.qz, I.qw, sh));
    h.front = dot(r.d, qrot<float>(I.qx, I.qy, I.qz, I.qw, geo)) < 0;
    if (!h.front) h.n = -h.n;
    h.u = w0 * A.u + ba * B.u + bb * C.u;  // deferred:801-803
    h.v = w0 * A.v + ba * B.v + bb * C.v;
    h.prim = (best - I.indexBase) / 3u;
    h.alpha = ba;
    h.beta = bb;
    return true;
}

// OccludedMesh, deferred:812-854.
inline bool occluded_mesh(const Scene &S, const ae_object &obj, const Ray<float> &r, float tn, float tf) {
    const ae_instance &I = S.instances[obj.instanceIndex];
    Ray<float> L;
    to_local(I, r, L);
    const Vf invd = 1.0f / L.d;
    int stack[64];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
        const ae_bvh_node &n = S.blas[I.blasBase + uint32_t(stack[--sp])];
        if (!slab(L.o, invd, n, tn, tf)) continue;
        if (n.count > 0) {
            for (int i = 0; i < n.count; i++) {
                const uint32_t base = I.indexBase + uint32_t(n.left + i) * 3u;
                float t, a, b;
                Vf g;
                if (hit_mesh_triangle(L, tn, tf, vpos<float>(S.vertices[I.vertexBase + S.indices[base]]),
                                      vpos<float>(S.vertices[I.vertexBase + S.indices[base + 1]]),
                                      vpos<float>(S.vertices[I.vertexBase + S.indices[base + 2]]), t, a, b, g))
                    return true;
            }
        } else {
            stack[sp++] = n.left;
            stack[sp++] = n.right;
        }
    }
    return false;
}

// IsRasterProxy, deferred:1011-1017.
inline bool raster_proxy(const ae_object &o) {
    return o.shapeType == AE_SHAPE_BOX && o.colorType != AE_MAT_ISOTROPIC && o.textureID == AE_NO_TEXTURE &&
           o.rotation == 0.0f;
}

// HitObject as deferred.comp dispatches it (its HitMesh is the ordered one).
inline bool hit_object_d(const Scene &S, const ae_object &o, const Ray<float> &r, float tn, float tf, Hit<float> &h,
                         Rng &rng) {
    if (o.colorType == AE_MAT_ISOTROPIC) return hit_volume(o, r, tn, tf, h, rng);
    switch (o.shapeType) {
    case AE_SHAPE_SPHERE: return hit_sphere(o, r, tn, tf, h);
    case AE_SHAPE_QUAD: return hit_planar(o, r, tn, tf, h, false);
    case AE_SHAPE_TRIANGLE: return hit_planar(o, r, tn, tf, h, true);
    case AE_SHAPE_MESH: return hit_mesh_ordered(S, o, r, tn, tf, h);
    default: return hit_box(o, r, tn, tf, h);
    }
}

// TraverseBVHBounded, deferred:1027-1099.
inline bool traverse_bounded(const Scene &S, const Ray<float> &r, float tn, float far_limit, bool skip, Hit<float> &out,
                             Rng &rng) {
    if (S.n_nodes == 0) return false;
    const Vf inv = 1.0f / r.d;
    int stack[64];
    int sp = 0;
    stack[sp++] = 0;
    bool found = false;
    float tf = far_limit;
    while (sp > 0) {
        const ae_bvh_node &n = S.tlas[stack[--sp]];
        if (!slab(r.o, inv, n, tn, tf)) continue;
        if (n.count > 0) {
            for (int i = 0; i < n.count; i++) {
                const uint32_t slot = uint32_t(n.left + i);
                const ae_object &o = S.objects[slot];
                if (skip && (o.shapeType == AE_SHAPE_MESH || raster_proxy(o))) continue;
                Hit<float> h;
                if (hit_object_d(S, o, r, tn, tf, h, rng)) {
                    tf = h.t;
                    h.obj = &o;
                    h.slot = slot;
                    out = h;
                    found = true;
                }
            }
        } else {
            const float tl = aabb_entry(r.o, inv, S.tlas[n.left], tn, tf);
            const float tr = aabb_entry(r.o, inv, S.tlas[n.right], tn, tf);
            const bool lf = tl <= tr;
            if (M<float>::fmax(tl, tr) < 1e30f) stack[sp++] = lf ? n.right : n.left;
            if (M<float>::fmin(tl, tr) < 1e30f) stack[sp++] = lf ? n.left : n.right;
        }
    }
    return found;
}

// Occluded, deferred:1115-1171.
inline bool occluded(const Scene &S, const Ray<float> &r, float tn, float tf, Rng &rng) {
    if (S.n_nodes == 0) return false;
    const Vf inv = 1.0f / r.d;
    int stack[64];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
        const ae_bvh_node &n = S.tlas[stack[--sp]];
        if (!slab(r.o, inv, n, tn, tf)) continue;
        if (n.count > 0) {
            for (int i = 0; i < n.count; i++) {
                const ae_object &o = S.objects[n.left + i];
                if (o.colorType == AE_MAT_DIELECTRIC || o.colorType == AE_MAT_DIFFUSE_LIGHT) continue;
                if (o.shapeType == AE_SHAPE_MESH) {
                    if (occluded_mesh(S, o, r, tn, tf)) return true;
                    continue;
                }
                Hit<float> h;
                if (hit_object_d(S, o, r, tn, tf, h, rng)) return true;
            }
        } else {
            stack[sp++] = n.left;
            stack[sp++] = n.right;
        }
    }
    return false;
}

// The deferred Hit: geometry plus the (possibly G-buffer) albedo it shades with.
struct DSurf {
    Hit<float> h;
    Vf albedo;  // Object.Albedo (the G-buffer's for raster surfaces)
    Vf surf;    // SurfaceAlbedo (deferred:1194-1203)
    const ae_object *obj = nullptr;
};

// CalculateDirectLight (deferred:1376-1446) + ClampedDirectLight (1556-1569).
inline Vf clamped_direct(const Scene &S, const DSurf &s, float time, Rng &rng) {
    Vf acc = v3<float>(0, 0, 0);
    for (uint32_t i = 0; i < S.n_lights; i++) {
        const ae_object &L = S.objects[S.lights[i]];
        Vf lp;
        float omega;
        sample_light(L, s.h.p, lp, omega, rng);
        if (omega <= 0) continue;
        Vf sd = lp - s.h.p;
        const float dist = len(sd);
        if (dist <= 1e-6f) continue;
        sd = sd / dist;
        const float ct = dot(s.h.n, sd);
        if (ct <= 0) continue;
        Ray<float> sr;
        sr.o = s.h.p + s.h.n * 0.001f;
        sr.d = sd;
        sr.time = time;
        if (!occluded(S, sr, 0.001f, dist - 0.001f, rng)) {
            const Vf rad = float(L.emission) * albedo<float>(L);
            acc = acc + s.surf * rad * ct * omega;
        }
    }
    const float luma = maxc(acc);
    if (luma > 8.0f) acc = acc * (8.0f / luma);
    return acc;
}

inline DSurf surf_of(const Scene &S, const Hit<float> &h) {
    DSurf s;
    s.h = h;
    s.obj = h.obj;
    s.albedo = albedo<float>(*h.obj);
    s.surf = surface_albedo(S, h);
    return s;
}

// GetBounce on a deferred surface (deferred:1219-1288).
inline bool bounce_d(const Ray<float> &r, const DSurf &s, Vf &dir, Rng &rng) { return bounce(r, s.h, dir, rng); }

// TraceIndirect, deferred:1575-1646.
inline Vf trace_indirect(const Scene &S, const ae_config &c, const Ray<float> &primary, const DSurf &surf, Rng &rng) {
    Vf bd;
    if (!bounce_d(primary, surf, bd, rng)) return v3<float>(0, 0, 0);
    Ray<float> ray;
    ray.d = nrm(bd);
    const float s0 = dot(ray.d, surf.h.n) < 0 ? -1.0f : 1.0f;
    ray.o = surf.h.p + surf.h.n * (0.001f * s0);
    ray.time = primary.time;
    Vf thr = surf.obj->colorType != AE_MAT_DIELECTRIC ? surf.surf : v3<float>(1, 1, 1);
    Vf acc = v3<float>(0, 0, 0);
    const Vf sky = v3<float>(c.sky_r, c.sky_g, c.sky_b);
    for (uint32_t b = 1; b < c.depth; b++) {
        Hit<float> h;
        if (!traverse_bounded(S, ray, 0.001f, 1000000.0f, false, h, rng)) {
            acc = acc + thr * sky;
            break;
        }
        if (h.obj->colorType == AE_MAT_DIFFUSE_LIGHT) {
            acc = acc + thr * (float(h.obj->emission) * albedo<float>(*h.obj));
            break;
        }
        const DSurf s = surf_of(S, h);
        if (h.obj->colorType == AE_MAT_LAMBERTIAN) acc = acc + thr * clamped_direct(S, s, ray.time, rng);
        Vf nx;
        if (!bounce(ray, h, nx, rng)) break;
        ray.d = nrm(nx);
        const float sg = dot(ray.d, h.n) < 0 ? -1.0f : 1.0f;
        ray.o = h.p + h.n * (0.001f * sg);
        if (h.obj->colorType != AE_MAT_DIELECTRIC) thr = thr * s.surf;
        float p = maxc(thr);
        p = M<float>::fmin(M<float>::fmax(p, 0.1f), 1.0f);
        if (rng.next<float>() > p) break;
        thr = thr / p;
    }
    return acc;
}

struct Planes {  // all W*H texels; albedo as float4 = byte/255
    const float *gpos, *gnrm, *galb, *gdepth;
    const float *prev_img, *prev_geo;
    float *img, *display, *reduced, *cur_geo;
    uint32_t red_w, red_h;
};

inline const float *at4(const float *p, uint32_t w, uint32_t x, uint32_t y) { return p + 4 * (size_t(y) * w + x); }

// CurrentRotation / PreviousRotation / PreviousPosition, deferred:1759-1793.
inline Vf previous_position(const Scene &S, const ae_object &o, Vf p) {
    float qx = 0, qy = 0, qz = 0, qw = 1;
    if (o.shapeType == AE_SHAPE_MESH) {
        const ae_instance &I = S.instances[o.instanceIndex];
        qx = I.qx; qy = I.qy; qz = I.qz; qw = I.qw;
    } else if (o.shapeType == AE_SHAPE_SPHERE || o.shapeType == AE_SHAPE_BOX) {
        const float half = 0.5f * o.rotation;
        qy = M<float>::sin(half);
        qw = M<float>::cos(half);
    }
    const Vf local = qrot<float>(-qx, -qy, -qz, qw, p - pos<float>(o));
    const Vf v = v3<float>(o.prevRotX, o.prevRotY, o.prevRotZ);
    const float w = M<float>::sqrt(M<float>::fmax(0.0f, 1.0f - dot(v, v)));
    return qrot<float>(v.x, v.y, v.z, w, local) + pos2<float>(o);
}

// ReprojectHistory, deferred:1810-1875 (same as upsample:218-278).
inline void reproject(const ae_config &c, uint32_t px, uint32_t py, Vf color, bool surface, Vf position, Vf prev_pos,
                      Vf normal, bool vd, const float *prev_img, const float *prev_geo, Vf &result, float &count) {
    const uint32_t W = c.width, H = c.height;
    int hx = int(px), hy = int(py);
    bool valid = c.historyReset == 0;
    const Vf src = v3<float>(c.source_x, c.source_y, c.source_z);
    if (valid && c.cameraMoved != 0) {
        valid = false;
        if (surface) {
            const float v[4] = {prev_pos.x, prev_pos.y, prev_pos.z, 1.0f};
            float clip[4];
            for (int r = 0; r < 4; r++) {
                const float *m = c.prevViewProj + 4 * r;
                clip[r] = m[0] * v[0] + m[1] * v[1] + m[2] * v[2] + m[3] * v[3];
            }
            if (clip[3] > 0) {
                const float ux = clip[0] / clip[3] * 0.5f + 0.5f;
                const float uy = clip[1] / clip[3] * -0.5f + 0.5f;
                const float fx = std::floor(ux * float(W)), fy = std::floor(uy * float(H));
                hx = int(std::fmax(std::fmin(fx, 2.0e9f), -2.0e9f));
                hy = int(std::fmax(std::fmin(fy, 2.0e9f), -2.0e9f));
                if (hx >= 0 && hy >= 0 && hx < int(W) && hy < int(H)) {
                    const float *pg = at4(prev_geo, W, hx, hy);
                    const Vf pp = v3<float>(pg[0], pg[1], pg[2]);
                    const float plane = std::fabs(dot(pp - prev_pos, normal));
                    const float tol = 0.01f * len(position - src) + 0.01f;
                    const float fp = len(position - src) * 2.0f * M<float>::tan(ae::radians(c.fov * 0.5f)) / float(H);
                    const float facing = M<float>::fmax(std::fabs(dot(normal, nrm(src - position))), 0.33f);
                    const float drift = len(pp - prev_pos);
                    valid = pg[3] > 0 && plane < tol && drift < M<float>::fmax(2.5f * fp / facing, 0.01f);
                }
            }
        }
    }
    if (!valid) {
        count = 1.0f;
        result = color;
        return;
    }
    const float prev_count = std::fabs(at4(prev_geo, W, hx, hy)[3]);
    const float moving = vd ? M<float>::fmin(c.historyCap, 4.0f) : c.historyCap;
    const float cap = c.cameraMoved != 0 ? moving : 1e7f;
    count = M<float>::fmin(prev_count + 1.0f, cap);
    const float *pi = at4(prev_img, W, hx, hy);
    const Vf prev = v3<float>(pi[0], pi[1], pi[2]);
    result = prev + (1.0f / count) * (color - prev);
}

// TracedTexel, deferred:1742-1747.
inline void traced_texel(const ae_config &c, uint32_t cx, uint32_t cy, uint32_t &tx, uint32_t &ty) {
    static const float off[4][2] = {{0.0f, 0.0f}, {0.5f, 0.5f}, {0.5f, 0.0f}, {0.0f, 0.5f}};
    const uint32_t k = c.frameIndex % 4u;
    const float fx = std::floor((float(cx) + off[k][0]) / c.traceScale);
    const float fy = std::floor((float(cy) + off[k][1]) / c.traceScale);
    tx = std::min(uint32_t(fx), c.width - 1);
    ty = std::min(uint32_t(fy), c.height - 1);
}

inline void put4(float *p, uint32_t w, uint32_t x, uint32_t y, Vf v, float a) {
    float *q = p + 4 * (size_t(y) * w + x);
    q[0] = v.x; q[1] = v.y; q[2] = v.z; q[3] = a;
}

// ResolvePrimary with HitFromGBuffer, deferred:1452-1548: 0 sky, 1 raster, 2 analytic.
inline int resolve_primary(const Scene &S, const ae_config &c, const Planes &P, uint32_t x, uint32_t y,
                           const Ray<float> &primary, Rng &rng, DSurf &hit) {
    const uint32_t W = c.width;
    DSurf raster;
    bool has_raster = false;
    float far_limit = 1000000.0f;
    const float *pn = at4(P.gnrm, W, x, y);
    if (!(pn[3] < 0.5f)) {
        const float *pp = at4(P.gpos, W, x, y);
        const uint32_t slot = uint32_t(pp[3] + 0.5f);
        if (slot < S.n_objects) {
            raster.obj = &S.objects[slot];
            raster.h.obj = raster.obj;
            raster.h.slot = slot;
            raster.h.p = v3<float>(pp[0], pp[1], pp[2]);
            raster.h.n = nrm(v3<float>(pn[0], pn[1], pn[2]));
            const float *pa = at4(P.galb, W, x, y);
            raster.albedo = v3<float>(pa[0], pa[1], pa[2]);
            raster.surf = raster.albedo;  // HitFromGBuffer clears TextureID (deferred:1477-1480)
            raster.h.front = dot(primary.d, raster.h.n) < 0;
            if (!raster.h.front) raster.h.n = -raster.h.n;
            raster.h.t = len(raster.h.p - primary.o);
            far_limit = raster.h.t;
            has_raster = true;
        }
    }
    Hit<float> ah;
    if (traverse_bounded(S, primary, 0.001f, far_limit, true, ah, rng)) {
        hit = surf_of(S, ah);
        return 2;
    }
    if (has_raster) {
        hit = raster;
        return 1;
    }
    return 0;
}

// MaterialFalseColour, deferred:1652-1663.
inline Vf false_colour(uint32_t t) {
    switch (t) {
    case AE_MAT_LAMBERTIAN: return v3<float>(0.55f, 0.55f, 0.55f);
    case AE_MAT_METAL: return v3<float>(1.0f, 0.75f, 0.1f);
    case AE_MAT_DIELECTRIC: return v3<float>(0.1f, 0.85f, 1.0f);
    case AE_MAT_DIFFUSE_LIGHT: return v3<float>(1.0f, 1.0f, 1.0f);
    case AE_MAT_ISOTROPIC: return v3<float>(0.7f, 0.3f, 1.0f);
    default: return v3<float>(1.0f, 0.0f, 1.0f);
    }
}

// DebugColour, deferred:1667-1722 (with WorldFromDepth, 1503-1514).
inline Vf debug_colour(const Scene &S, const ae_config &c, const Planes &P, uint32_t x, uint32_t y,
                       const Ray<float> &primary, Rng &rng, const Camera<float> &K) {
    const uint32_t W = c.width;
    const float *pn = at4(P.gnrm, W, x, y);
    const bool covered = pn[3] >= 0.5f;
    const Vf bg = v3<float>(0, 0, 0);
    if (c.debugView == 1) {
        const float *pa = at4(P.galb, W, x, y);
        return covered ? v3<float>(pa[0], pa[1], pa[2]) : bg;
    }
    if (c.debugView == 2) return covered ? v3<float>(pn[0], pn[1], pn[2]) * 0.5f + v3<float>(0.5f, 0.5f, 0.5f) : bg;
    if (c.debugView == 3) {
        if (!covered) return bg;
        const float *pp = at4(P.gpos, W, x, y);
        const Vf q = v3<float>(pp[0], pp[1], pp[2]) / 100.0f;
        return v3<float>(ae::fracf(q.x), ae::fracf(q.y), ae::fracf(q.z));
    }
    if (c.debugView == 6) {
        if (!covered) return v3<float>(0.0f, 0.0f, 0.2f);
        const float *pp = at4(P.gpos, W, x, y);
        const Vf stored = v3<float>(pp[0], pp[1], pp[2]);
        const float dd = P.gdepth[size_t(y) * W + x];
        const float vz = (c.zNear * c.zFar) / (c.zFar + dd * (c.zNear - c.zFar));
        const Vf fwd = -nrm(K.src - v3<float>(c.target_x, c.target_y, c.target_z));
        const float t = vz / dot(primary.d, fwd);
        const Vf rebuilt = K.src + primary.d * t;
        const float rel = len(rebuilt - stored) / M<float>::fmax(len(stored - K.src), 1e-4f);
        const float v = rel * 100.0f;
        return v3<float>(v, v, v);
    }
    DSurf hit;
    const int source = resolve_primary(S, c, P, x, y, primary, rng, hit);
    if (c.debugView == 4) return source != 0 ? false_colour(hit.obj->colorType) : bg;
    if (source == 1) return v3<float>(0.1f, 0.8f, 0.2f);
    if (source == 2) return v3<float>(0.85f, 0.15f, 0.1f);
    return v3<float>(0.1f, 0.15f, 0.5f);
}

// main, deferred:1879-2010 (final view).
inline void deferred_cell(const Scene &S, const ae_config &c, const Planes &P, uint32_t cx, uint32_t cy) {
    const bool reduced = c.traceScale < 1.0f;
    uint32_t x = cx, y = cy;
    if (reduced) traced_texel(c, cx, cy, x, y);
    const uint32_t W = c.width;
    if (c.displayOnly) {
        if (!reduced) {
            const float *a = at4(P.img, W, x, y);
            put4(P.display, W, x, y, srgb(aces(v3<float>(a[0], a[1], a[2]) * c.exposure)), 1.0f);
        }
        return;
    }
    Rng rng{x + y * c.width + c.frameIndex * c.width * c.height + 1u};
    const Camera<float> K = camera<float>(c);
    const Vf sample = K.p0 + (float(x) + c.jitter_x) * K.pu + (float(y) + c.jitter_y) * K.pv;
    Ray<float> primary;
    primary.o = K.src;
    primary.d = nrm(sample - K.src);
    primary.time = rng.next<float>();
    if (c.debugView != 0) {
        put4(P.display, W, x, y, debug_colour(S, c, P, x, y, primary, rng, K), 1.0f);
        return;
    }
    // ResolvePrimary + HitFromGBuffer, deferred:1452-1548.
    DSurf raster;
    bool has_raster = false;
    float far_limit = 1000000.0f;
    const float *pn = at4(P.gnrm, W, x, y);
    if (!(pn[3] < 0.5f)) {
        const float *pp = at4(P.gpos, W, x, y);
        const uint32_t slot = uint32_t(pp[3] + 0.5f);
        if (slot < S.n_objects) {
            raster.obj = &S.objects[slot];
            raster.h.obj = raster.obj;
            raster.h.slot = slot;
            raster.h.p = v3<float>(pp[0], pp[1], pp[2]);
            raster.h.n = nrm(v3<float>(pn[0], pn[1], pn[2]));
            const float *pa = at4(P.galb, W, x, y);
            raster.albedo = v3<float>(pa[0], pa[1], pa[2]);
            raster.surf = raster.albedo;  // HitFromGBuffer clears TextureID (deferred:1477-1480)
            raster.h.front = dot(primary.d, raster.h.n) < 0;
            if (!raster.h.front) raster.h.n = -raster.h.n;
            raster.h.t = len(raster.h.p - K.src);
            far_limit = raster.h.t;
            has_raster = true;
        }
    }
    DSurf hit;
    int source = 0;
    Hit<float> ah;
    if (traverse_bounded(S, primary, 0.001f, far_limit, true, ah, rng)) {
        hit = surf_of(S, ah);
        source = 2;
    } else if (has_raster) {
        hit = raster;
        source = 1;
    }
    Vf color = v3<float>(0, 0, 0);
    if (source == 0) {
        color = v3<float>(c.sky_r, c.sky_g, c.sky_b);
    } else if (hit.obj->colorType == AE_MAT_DIFFUSE_LIGHT) {
        color = float(hit.obj->emission) * hit.albedo;
    } else {
        const uint32_t per = c.batches ? c.samples / c.batches : c.samples;
        const uint32_t spp = per > 1u ? per : 1u;
        for (uint32_t s = 0; s < spp; s++) {
            if (hit.obj->colorType == AE_MAT_LAMBERTIAN) color = color + clamped_direct(S, hit, primary.time, rng);
            color = color + trace_indirect(S, c, primary, hit, rng);
        }
        color = color / float(spp);
    }
    if (reduced) {
        const bool demod = source == 1 && hit.obj->colorType != AE_MAT_DIELECTRIC;
        Vf alb = v3<float>(1, 1, 1);
        if (demod) alb = vmax(hit.surf, v3<float>(0.01f, 0.01f, 0.01f));
        put4(P.reduced, P.red_w, cx, cy, color / alb, demod ? 1.0f : 0.0f);
        return;
    }
    const bool surface = source != 0;
    const bool vd = surface && (hit.obj->colorType == AE_MAT_METAL || hit.obj->colorType == AE_MAT_DIELECTRIC);
    const Vf hp = surface ? hit.h.p : v3<float>(0, 0, 0);
    const Vf prev = surface ? previous_position(S, *hit.obj, hit.h.p) : hp;
    Vf acc;
    float hl;
    reproject(c, x, y, color, surface, hp, prev, surface ? hit.h.n : v3<float>(0, 0, 0), vd, P.prev_img, P.prev_geo, acc,
              hl);
    put4(P.img, W, x, y, acc, 1.0f);
    put4(P.cur_geo, W, x, y, hp, surface ? hl : -hl);
    put4(P.display, W, x, y, srgb(aces(acc * c.exposure)), 1.0f);
}

// main, upsample:280-390.
inline void upsample_pixel(const Scene &S, const ae_config &c, const Planes &P, uint32_t x, uint32_t y) {
    const uint32_t W = c.width;
    if (c.displayOnly) {
        const float *a = at4(P.img, W, x, y);
        put4(P.display, W, x, y, srgb(aces(v3<float>(a[0], a[1], a[2]) * c.exposure)), 1.0f);
        return;
    }
    const Vf src = v3<float>(c.source_x, c.source_y, c.source_z);
    const int cmx = int(P.red_w) - 1, cmy = int(P.red_h) - 1;
    const float *np = at4(P.gnrm, W, x, y);
    const bool covp = np[3] > 0.5f;
    const float *gp = at4(P.gpos, W, x, y);
    const float dp = len(v3<float>(gp[0], gp[1], gp[2]) - src);
    const float *ap = at4(P.galb, W, x, y);
    const Vf albp = v3<float>(ap[0], ap[1], ap[2]);
    const float cpx = (float(x) + 0.5f) * c.traceScale - 0.5f, cpy = (float(y) + 0.5f) * c.traceScale - 0.5f;
    const int bx = int(std::floor(cpx)), by = int(std::floor(cpy));
    Vf sum = v3<float>(0, 0, 0), nearest = v3<float>(0, 0, 0);
    float wsum = 0, nd = 1e30f;
    for (int j = 0; j < 2; j++)
        for (int i = 0; i < 2; i++) {
            const uint32_t cx = uint32_t(std::min(std::max(bx + i, 0), cmx)), cy = uint32_t(std::min(std::max(by + j, 0), cmy));
            uint32_t tx, ty;
            traced_texel(c, cx, cy, tx, ty);
            const float *lit = at4(P.reduced, P.red_w, cx, cy);
            const float *nt = at4(P.gnrm, W, tx, ty);
            const bool covt = nt[3] > 0.5f;
            Vf alb = albp;
            if (!covp) { const float *at = at4(P.galb, W, tx, ty); alb = v3<float>(at[0], at[1], at[2]); }
            const Vf l = v3<float>(lit[0], lit[1], lit[2]);
            const Vf rad = lit[3] > 0.5f ? l * alb : l;
            const float ox = float(tx) - float(x), oy = float(ty) - float(y);
            const float d2 = ox * ox + oy * oy;
            if (d2 < nd) { nd = d2; nearest = rad; }
            float w = ae::expf_(-d2 * c.traceScale * c.traceScale);
            if (covt != covp) {
                w = 0;
            } else if (covp) {
                const float *gt = at4(P.gpos, W, tx, ty);
                const float dt = len(v3<float>(gt[0], gt[1], gt[2]) - src);
                w *= ae::expf_(-std::fabs(dp - dt) / (0.01f * dp + 0.001f));
                w *= ae::powf_(sat(np[0] * nt[0] + np[1] * nt[1] + np[2] * nt[2]), 32.0f);
            }
            sum = sum + w * rad;
            wsum += w;
        }
    const Vf color = wsum > 1e-4f ? sum / wsum : nearest;
    const Vf posp = v3<float>(gp[0], gp[1], gp[2]);
    const bool vd = covp && ap[3] < 0.5f;
    Vf prev = posp;
    if (covp) {
        const uint32_t slot = uint32_t(gp[3]);
        if (slot < S.n_objects) prev = previous_position(S, S.objects[slot], posp);
    }
    Vf acc;
    float hl;
    reproject(c, x, y, color, covp, posp, prev, v3<float>(np[0], np[1], np[2]), vd, P.prev_img, P.prev_geo, acc, hl);
    put4(P.img, W, x, y, acc, 1.0f);
    put4(P.cur_geo, W, x, y, posp, covp ? hl : -hl);
    put4(P.display, W, x, y, srgb(aces(acc * c.exposure)), 1.0f);
}

}  // namespace oracle

extern "C" {

int oracle_deferred(const Scene *S, const ae_config *c, const Planes *P, int threads) {
    if (threads > 0) omp_set_num_threads(threads);
    const bool reduced = c->traceScale < 1.0f;
    const uint32_t ew = reduced ? P->red_w : c->width, eh = reduced ? P->red_h : c->height;
#pragma omp parallel for schedule(dynamic, 1)
    for (int y = 0; y < int(eh); y++)
        for (uint32_t x = 0; x < ew; x++) deferred_cell(*S, *c, *P, x, uint32_t(y));
    return 0;
}

int oracle_upsample(const Scene *S, const ae_config *c, const Planes *P, int threads) {
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 1)
    for (int y = 0; y < int(c->height); y++)
        for (uint32_t x = 0; x < c->width; x++) upsample_pixel(*S, *c, *P, x, uint32_t(y));
    return 0;
}

}  // extern "C"

// The library's ray-cast G-buffer (in place of gbuffer.vert/frag.hlsl): the
// closest hit through pixel centre + jitter over what the raster pass draws
// (meshes and raster proxies), by the compute-only walk.  Planes as the
// kernel writes them: position (w = slot), outward normal (w = coverage),
// albedo bytes (a = 0 view-dependent), depth.
extern "C" int oracle_gbuffer(const oracle::Scene *S, const ae_config *c, float *gpos, float *gnrm, uint8_t *galb,
                              float *gdepth, int threads) {
    using namespace oracle;
    if (threads > 0) omp_set_num_threads(threads);
    const Camera<float> K = camera<float>(*c);
    const Vf fwd = -nrm(K.src - v3<float>(c->target_x, c->target_y, c->target_z));
#pragma omp parallel for schedule(dynamic, 4)
    for (int y = 0; y < int(c->height); y++)
        for (uint32_t x = 0; x < c->width; x++) {
            const size_t px = size_t(y) * c->width + x;
            const Vf sample = K.p0 + (float(x) + c->jitter_x) * K.pu + (float(uint32_t(y)) + c->jitter_y) * K.pv;
            Ray<float> r;
            r.o = K.src;
            r.d = nrm(sample - K.src);
            r.time = 0;
            float *P = gpos + 4 * px, *N = gnrm + 4 * px;
            uint8_t *A = galb + 4 * px;
            P[0] = P[1] = P[2] = P[3] = 0;
            N[0] = N[1] = N[2] = N[3] = 0;
            A[0] = A[1] = A[2] = A[3] = 0;
            gdepth[px] = 1.0f;
            if (S->n_nodes == 0) continue;
            const Vf inv = 1.0f / r.d;
            int stack[64];
            int sp = 0;
            stack[sp++] = 0;
            float tf = 1000000.0f;
            bool found = false;
            Hit<float> best;
            Rng rng{1u};
            while (sp > 0) {
                const ae_bvh_node &n = S->tlas[stack[--sp]];
                if (!slab(r.o, inv, n, 0.001f, tf)) continue;
                if (n.count > 0) {
                    for (int i = 0; i < n.count; i++) {
                        const uint32_t slot = uint32_t(n.left + i);
                        const ae_object &o = S->objects[slot];
                        Hit<float> h;
                        bool hit = false;
                        if (o.shapeType == AE_SHAPE_MESH) hit = hit_mesh(*S, o, r, 0.001f, tf, h, nullptr);
                        else if (raster_proxy(o)) hit = hit_box(o, r, 0.001f, tf, h);
                        if (hit) {
                            tf = h.t;
                            h.obj = &o;
                            h.slot = slot;
                            best = h;
                            found = true;
                        }
                    }
                } else {
                    stack[sp++] = n.left;
                    stack[sp++] = n.right;
                }
            }
            (void)rng;
            if (!found) continue;
            const Vf nn = best.front ? best.n : -best.n;
            P[0] = best.p.x; P[1] = best.p.y; P[2] = best.p.z; P[3] = float(best.slot);
            N[0] = nn.x; N[1] = nn.y; N[2] = nn.z; N[3] = 1.0f;
            const ae_object &o = *best.obj;
            // SurfaceBlock's albedo (gbuffer.frag:44-50), textured at the hit's UV.
            const Vf sa = surface_albedo(*S, best);
            const float al[3] = {sa.x, sa.y, sa.z};
            for (int k = 0; k < 3; k++) A[k] = uint8_t(int(std::rint(std::fmin(std::fmax(al[k], 0.0f), 1.0f) * 255.0f)));
            A[3] = (o.colorType == AE_MAT_METAL || o.colorType == AE_MAT_DIELECTRIC) ? 0 : 255;
            const float vz = dot(best.p - r.o, fwd);
            gdepth[px] = c->zFar * (c->zNear - vz) / ((c->zNear - c->zFar) * vz);
        }
    return 0;
}

// Any hit per ray with deferred.comp's rules (Occluded, deferred:1115-1171).
extern "C" int oracle_any_hit(const oracle::Scene *S, const ae_ray *rays, const float *tmax, uint32_t n, uint8_t *out,
                              int threads) {
    using namespace oracle;
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t i = 0; i < int64_t(n); i++) {
        Ray<float> r;
        r.o = v3<float>(rays[i].ox, rays[i].oy, rays[i].oz);
        r.d = v3<float>(rays[i].dx, rays[i].dy, rays[i].dz);
        r.time = rays[i].time;
        Rng rng{1u};
        out[i] = occluded(*S, r, rays[i].tnear, tmax[i], rng) ? 1 : 0;
    }
    return 0;
}
