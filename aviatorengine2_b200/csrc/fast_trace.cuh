// fast_trace.cuh - the optimised closest-hit traversal: data layout (4-wide
// quantised BLAS, leaf-ordered triangle records, per-instance records) and the
// device walk, shared by the closest-hit entry points and the wavefront path
// tracer.  See fast.cu for how the structures are built and why the results
// match the reference's walk.
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "context.h"
#include "trace_common.cuh"

namespace ae {

struct QNode {               // 64 B
    float ox, oy, oz;        // node box minimum
    int8_t ex, ey, ez;       // child box scale 2^e per axis
    uint8_t nchild;          // children in use (2..4)
    uint8_t lo[3][4];        // [axis][child]
    uint8_t hi[3][4];
    uint32_t child[4];       // interior: node index; leaf: leaf_ref(first, count)
    uint32_t pad[2];
};
static_assert(sizeof(QNode) == 64, "QNode must be 64 bytes");
constexpr uint32_t kLeafBit = 0x80000000u;
// A leaf reference: bit 31 set, primitive count in bits 24-30 (1..127), first
// slot in bits 0-23.  prepare_fast refuses meshes outside those limits.
constexpr uint32_t kMaxLeafFirst = 1u << 24;
constexpr uint32_t kMaxLeafCount = 127u;
__host__ __device__ inline uint32_t leaf_ref(uint32_t first, uint32_t count) { return kLeafBit | (count << 24) | first; }
__host__ __device__ inline uint32_t leaf_first(uint32_t ref) { return ref & 0x00ffffffu; }
__host__ __device__ inline uint32_t leaf_count(uint32_t ref) { return (ref >> 24) & 0x7fu; }

struct FastInst {            // 48 B
    float px, py, pz, scale;
    float qx, qy, qz, qw;
    uint32_t root;           // QNode index of the mesh root, or a leaf ref
    uint32_t tri_base;       // first triangle record of the mesh
    uint32_t pad[2];
};
static_assert(sizeof(FastInst) == 48, "FastInst must be 48 bytes");

struct FastScene {
    DevBuf<QNode> nodes;
    DevBuf<float4> tris;     // 3 float4 per triangle
    DevBuf<FastInst> inst;
    DevBuf<uint4> obj_meta;  // per object slot: shape | material << 8, instance
    DevBuf<uint4> shade16;   // precision form: FP16 normals and UVs, 2 per triangle
    uint32_t shade16_tris = 0;
    // Ray counters of the batch walker (k_closest_walk), one per launch in
    // flight: a ring, so launches on different streams never share one.
    static constexpr uint32_t kWalkCounters = 64;
    DevBuf<uint32_t> walk_next;
    uint32_t walk_pos = 0;
    uint32_t n_nodes = 0, n_tris = 0;
    int max_stack = 0;
    uint64_t geometry_key = ~0ull, scene_key = ~0ull;
    bool has_volumes = false;
    // host_nodes / host_tris grew and are not on the device yet (an upload
    // that failed is retried by the next prepare_fast)
    bool geometry_dirty = false;
    // per distinct mesh (vertexBase, indexBase, triangleCount, blasBase)
    std::map<std::tuple<uint32_t, uint32_t, uint32_t, uint32_t>, std::pair<uint32_t, uint32_t>> mesh_roots;
    std::vector<QNode> host_nodes;
    std::vector<float> host_tris;
};

// Traversal stack per thread: the first kSharedStack entries in shared
// memory, the rest (rarely reached: only along the deepest paths of the
// largest meshes) in a per-thread local array.  prepare_fast checks that no
// tree needs more than kFastStack entries.
constexpr int kSharedStack = 24;
constexpr int kLocalStack = 40;
constexpr int kFastStack = kSharedStack + kLocalStack;

// ---------------------------------------------------------------------------
// Device
// ---------------------------------------------------------------------------
struct FastView {
    const QNode *nodes;
    const float4 *tris;
    const FastInst *inst;
    const uint4 *meta;
};

// Best candidate so far with its visit rank (see the file comment).  A
// candidate ranks by (object rank, leaf rank, slot): object rank is
// (~first slot of its TLAS leaf) << 32 | object slot, leaf rank is ~first slot
// of its BLAS leaf; larger means visited later by the reference's walk.
struct Best {
    float t, alpha, beta;
    uint32_t object, prim;
    uint64_t orank;
    uint32_t lrank;
};
// Given a hit at t <= best.t (the tests reject t > far), keep it if nearer or
// equally near and later in the reference's visit order.
AE_DEV bool takes(const Best &b, float t, uint64_t orank, uint32_t lrank, uint32_t slot) {
    if (t < b.t) return true;
    if (orank != b.orank) return orank > b.orank;
    if (lrank != b.lrank) return lrank > b.lrank;
    return slot > b.prim;
}

// HitMeshTriangle (hybrid:564-598), correctly rounded; p1/p2 give e1/e2 by the
// same subtraction the reference performs.
AE_DEV bool tri_test_ref(f3 o, f3 d, float tn, float tf, const float4 &r0, const float4 &r1, const float4 &r2,
                         float &t, float &a, float &b) {
    const f3 p0 = mk(r0.x, r0.y, r0.z), p1 = mk(r0.w, r1.x, r1.y), p2 = mk(r1.z, r1.w, r2.x);
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
    return !(a < 0.0f || b < 0.0f || AE_ADD(a, b) > 1.0f);
}

// The watertight test (trace_common.cuh) over a 48-byte triangle record.
AE_DEV bool tri_test_wt(f3 o, const WtRay &W, float tn, float tf, const float4 &r0, const float4 &r1,
                        const float4 &r2, float &t, float &a, float &b) {
    return tri_wt(o, W, tn, tf, mk(r0.x, r0.y, r0.z), mk(r0.w, r1.x, r1.y), mk(r1.z, r1.w, r2.x), t, a, b);
}

// Relative widening of slab intervals in the optimised walk (entry scaled
// down, exit scaled up; t >= tnear > 0 on the entry side).
constexpr float kEntryShrink = 0.99999904632568359375f;  // 1 - 2^-20
constexpr float kExitGrow = 1.00000095367431640625f;     // 1 + 2^-20

// Byte k (0..3) of w as an exact float: the byte permute builds the bits
// 0x4B0000bb, which are 2^23 + bb, and the subtraction is exact.  Same value
// as float(bb), without a conversion on the XU pipe.
AE_DEV float byte_as_float(uint32_t w, int k) {
    const uint32_t bits = __byte_perm(w, 0x4B000000u, 0x7440u | uint32_t(k));
    return __fsub_rn(__uint_as_float(bits), 8388608.0f);
}

// Entry distance of the 4 quantised child boxes; an inverted slot or a miss
// yields +inf.  Computed as q * (s/d) + (o - p)/d per slab with a relative
// widening of 2^-20 on the exit side, which covers the rounding of this
// formulation (the decoded boxes already contain the exact ones).
//
// The near and far planes of each slab are picked once per node from the sign
// of the direction term: the rounded fma is monotone in q, so for a valid
// child (lo <= hi) the pick gives exactly min and max of the two plane
// distances, and the intervals are bit for bit those of the min/max form.
AE_DEV void child_hits(const QNode *nodep, f3 o, f3 inv, float tn, float tf, float tmin[4], uint32_t child[4]) {
    const float4 *p = reinterpret_cast<const float4 *>(nodep);
    const float4 w0 = __ldg(p), w1 = __ldg(p + 1), w2 = __ldg(p + 2), w3 = __ldg(p + 3);
    const uint32_t meta = __float_as_uint(w0.w);
    const int ex = int(int8_t(meta & 0xff)), ey = int(int8_t((meta >> 8) & 0xff)), ez = int(int8_t((meta >> 16) & 0xff));
    const float sx = __int_as_float((ex + 127) << 23), sy = __int_as_float((ey + 127) << 23),
                sz = __int_as_float((ez + 127) << 23);
    const float ix = sx * inv.x, iy = sy * inv.y, iz = sz * inv.z;
    const float bx = (w0.x - o.x) * inv.x, by = (w0.y - o.y) * inv.y, bz = (w0.z - o.z) * inv.z;
    const uint32_t lox = __float_as_uint(w1.x), loy = __float_as_uint(w1.y), loz = __float_as_uint(w1.z);
    const uint32_t hix = __float_as_uint(w1.w), hiy = __float_as_uint(w2.x), hiz = __float_as_uint(w2.y);
    // Near-plane and far-plane bytes per axis.
    const uint32_t nx = ix >= 0.0f ? lox : hix, fx = ix >= 0.0f ? hix : lox;
    const uint32_t ny = iy >= 0.0f ? loy : hiy, fy = iy >= 0.0f ? hiy : loy;
    const uint32_t nz = iz >= 0.0f ? loz : hiz, fz = iz >= 0.0f ? hiz : loz;
    // A slot is in use when its x range is not inverted (one byte-wise compare).
    const uint32_t valid = __vcmpleu4(lox, hix);
    child[0] = __float_as_uint(w2.z); child[1] = __float_as_uint(w2.w);
    child[2] = __float_as_uint(w3.x); child[3] = __float_as_uint(w3.y);
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const float t0x = fmaf(byte_as_float(nx, k), ix, bx), t1x = fmaf(byte_as_float(fx, k), ix, bx);
        const float t0y = fmaf(byte_as_float(ny, k), iy, by), t1y = fmaf(byte_as_float(fy, k), iy, by);
        const float t0z = fmaf(byte_as_float(nz, k), iz, bz), t1z = fmaf(byte_as_float(fz, k), iz, bz);
        const float lo = fmaxf(fmaxf(t0x, t0y), fmaxf(t0z, tn));
        const float hi = fminf(fminf(t1x, t1y), t1z);
        // Widened by 2^-20 relative on both sides: the interval computed here
        // then contains the exact one, so neither a closer hit nor one lying
        // on the box's face is pruned by rounding.
        const float lo_c = lo * kEntryShrink;
        const bool hit = ((valid >> (8 * k)) & 1u) && lo_c <= fminf(hi * kExitGrow, tf);
        tmin[k] = hit ? lo_c : __int_as_float(0x7f800000);
    }
}

// Safe reciprocal for slab tests: a zero component becomes a huge finite
// value of the same sign, so products stay finite (no 0 * inf).
AE_DEV float slab_inv(float x) { return fabsf(x) > 1e-20f ? 1.0f / x : copysignf(1e20f, x); }

// T (optional): touch counters - wide nodes in `blas`, 48-byte triangle
// records in `tris`.
template <bool WT, int SS = kSharedStack>
AE_DEV void trace_mesh(const FastView &V, const FastInst &I, uint32_t slot, uint64_t orank, f3 o, f3 d, float tn,
                       Best &best, uint2 *stk, int tid, int nthreads, Touch *T = nullptr) {
    // ToLocal (hybrid:534-543) exactly as the reference, so the local ray and
    // every triangle's t are bit-identical to the plain kernel's.
    f3 lo = quat_rotate(-I.qx, -I.qy, -I.qz, I.qw, o - mk(I.px, I.py, I.pz));
    f3 ld = quat_rotate(-I.qx, -I.qy, -I.qz, I.qw, d);
    if (I.scale != 0.0f && I.scale != 1.0f) {
        const float inv = AE_DIV(1.0f, I.scale);
        lo = lo * inv;
        ld = ld * inv;
    }
    const f3 inv = mk(slab_inv(ld.x), slab_inv(ld.y), slab_inv(ld.z));
    WtRay W;
    if (WT) W = wt_setup(ld);
    const float4 *tris = V.tris + size_t(I.tri_base) * 3;
    uint2 spill[kFastStack - SS];
    int sp = 0;
    uint32_t cur = I.root;
    for (;;) {
        if (cur & kLeafBit) {
            const uint32_t first = leaf_first(cur), cnt = leaf_count(cur);
            if (T) T->tris += cnt;
            for (uint32_t k = 0; k < cnt; k++) {
                const uint32_t s = first + k;
                const float4 *r = tris + size_t(s) * 3;
                const float4 r0 = __ldg(r), r1 = __ldg(r + 1), r2 = __ldg(r + 2);
                float t, a, b;
                const bool h = WT ? tri_test_wt(lo, W, tn, best.t, r0, r1, r2, t, a, b)
                                  : tri_test_ref(lo, ld, tn, best.t, r0, r1, r2, t, a, b);
                if (h && takes(best, t, orank, ~first, s)) {
                    best.t = t; best.alpha = a; best.beta = b;
                    best.object = slot; best.prim = s;
                    best.orank = orank; best.lrank = ~first;
                }
            }
        } else {
            float tm[4];
            uint32_t ch[4];
            if (T) T->blas++;
            child_hits(V.nodes + cur, lo, inv, tn, best.t, tm, ch);
            // Sort the four (distance, child) pairs, nearest first.
#define AE_SWAP(i, j)                                            \
    if (tm[j] < tm[i]) {                                         \
        const float tt = tm[i]; tm[i] = tm[j]; tm[j] = tt;       \
        const uint32_t cc = ch[i]; ch[i] = ch[j]; ch[j] = cc;    \
    }
            AE_SWAP(0, 1) AE_SWAP(2, 3) AE_SWAP(0, 2) AE_SWAP(1, 3) AE_SWAP(1, 2)
#undef AE_SWAP
            int nh = 0;
#pragma unroll
            for (int k = 0; k < 4; k++) nh += tm[k] != __int_as_float(0x7f800000) ? 1 : 0;
            if (nh > 0) {
                // Far hits onto the stack (farthest deepest), continue with the
                // nearest.  prepare_fast checked that the tree never needs more
                // than kFastStack entries; the bound check keeps that true for
                // any input.
                for (int k = nh - 1; k >= 1; k--) {
                    if (sp < SS) stk[sp * nthreads + tid] = make_uint2(ch[k], __float_as_uint(tm[k]));
                    else if (sp < kFastStack) spill[sp - SS] = make_uint2(ch[k], __float_as_uint(tm[k]));
                    sp = sp < kFastStack ? sp + 1 : sp;
                }
                cur = ch[0];
                continue;
            }
        }
        // Pop the next entry still no farther than the best hit.
        bool found = false;
        while (sp > 0) {
            sp--;
            const uint2 e = sp < SS ? stk[sp * nthreads + tid] : spill[sp - SS];
            if (__uint_as_float(e.y) <= best.t) {
                cur = e.x;
                found = true;
                break;
            }
        }
        if (!found) break;
    }
}

// Closest hit of one ray over the whole scene: TLAS (the reference's binary
// nodes, nearest child first), analytic objects by the reference intersectors,
// meshes by the 4-wide quantised BLAS.  `stk` is this thread's column of the
// block's shared-memory stack.  T (optional) counts the touches: TLAS nodes,
// object metadata records, instance records, wide BLAS nodes, triangle records.
template <bool WT, int SS = kSharedStack>
AE_DEV Best closest_fast(const DevScene &S, const FastView &V, f3 o, f3 d, float tn, float time, uint2 *stk, int tid,
                         int nt, Touch *T = nullptr) {
    Best best;
    best.t = kFarStart; best.alpha = 0.0f; best.beta = 0.0f;
    best.object = AE_MISS; best.prim = AE_MISS; best.orank = 0; best.lrank = 0;
    if (S.n_nodes == 0) return best;
    const f3 inv = mk(slab_inv(d.x), slab_inv(d.y), slab_inv(d.z));
    const f3 rinv = 1.0f / d;
    int tstack[kTlasStack];
    float tdist[kTlasStack];
    int sp = 0;
    NodeBox nb = load_node(S.tlas, 0);
    if (T) T->tlas++;
    bool live = slab_ref(o, rinv, nb.lo, nb.hi, tn, kFarStart);
    while (live) {
        if (nb.count > 0) {
            const uint32_t first = uint32_t(nb.left);
            for (int k = 0; k < nb.count; k++) {
                const uint32_t slot = first + uint32_t(k);
                const uint64_t orank = (uint64_t(~first) << 32) | slot;
                const uint4 m = __ldg(V.meta + slot);
                const uint32_t shape = m.x & 0xff;
                if (T) T->objects++;
                if (shape == AE_SHAPE_MESH) {
                    if (T) T->instances++;
                    const float4 *ip = reinterpret_cast<const float4 *>(V.inst + m.y);
                    const float4 a = __ldg(ip), b = __ldg(ip + 1), c = __ldg(ip + 2);
                    FastInst I;
                    I.px = a.x; I.py = a.y; I.pz = a.z; I.scale = a.w;
                    I.qx = b.x; I.qy = b.y; I.qz = b.z; I.qw = b.w;
                    I.root = __float_as_uint(c.x); I.tri_base = __float_as_uint(c.y);
                    trace_mesh<WT, SS>(V, I, slot, orank, o, d, tn, best, stk, tid, nt, T);
                } else {
                    DHit h;
                    const ae_object *obj = S.objects + slot;
                    bool hit;
                    if (shape == AE_SHAPE_SPHERE) hit = hit_sphere_ref(obj, o, d, time, tn, best.t, h);
                    else if (shape == AE_SHAPE_QUAD) hit = hit_planar_ref(obj, false, o, d, tn, best.t, h);
                    else if (shape == AE_SHAPE_TRIANGLE) hit = hit_planar_ref(obj, true, o, d, tn, best.t, h);
                    else hit = hit_box_ref(obj, o, d, tn, best.t, h);
                    if (hit && takes(best, h.t, orank, 0u, 0u)) {
                        best.t = h.t; best.alpha = h.alpha; best.beta = h.beta;
                        best.object = slot; best.prim = AE_MISS; best.orank = orank; best.lrank = 0;
                    }
                }
            }
        } else {
            const NodeBox L = load_node(S.tlas, uint32_t(nb.left)), R = load_node(S.tlas, uint32_t(nb.right));
            if (T) T->tlas += 2;
            const f3 lt0 = (L.lo - o) * inv, lt1 = (L.hi - o) * inv;
            const f3 rt0 = (R.lo - o) * inv, rt1 = (R.hi - o) * inv;
            const float lmin = fmaxf(fmaxf(fminf(lt0.x, lt1.x), fminf(lt0.y, lt1.y)), fmaxf(fminf(lt0.z, lt1.z), tn));
            const float lmax = fminf(fminf(fmaxf(lt0.x, lt1.x), fmaxf(lt0.y, lt1.y)), fmaxf(lt0.z, lt1.z));
            const float rmin = fmaxf(fmaxf(fminf(rt0.x, rt1.x), fminf(rt0.y, rt1.y)), fmaxf(fminf(rt0.z, rt1.z), tn));
            const float rmax = fminf(fminf(fmaxf(rt0.x, rt1.x), fmaxf(rt0.y, rt1.y)), fmaxf(rt0.z, rt1.z));
            const float lmin_c = lmin * kEntryShrink, rmin_c = rmin * kEntryShrink;
            const bool lh = lmin_c <= fminf(lmax * kExitGrow, best.t);
            const bool rh = rmin_c <= fminf(rmax * kExitGrow, best.t);
            if (lh && rh) {
                const bool lfirst = lmin <= rmin;
                if (sp < kTlasStack) {
                    tstack[sp] = lfirst ? nb.right : nb.left;
                    tdist[sp] = lfirst ? rmin_c : lmin_c;
                    sp++;
                }
                nb = lfirst ? L : R;
                continue;
            }
            if (lh) { nb = L; continue; }
            if (rh) { nb = R; continue; }
        }
        live = false;
        while (sp > 0) {
            sp--;
            if (tdist[sp] <= best.t) {
                nb = load_node(S.tlas, uint32_t(tstack[sp]));
                live = true;
                break;
            }
        }
    }
    return best;
}

}  // namespace ae
