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

// The instance-level tree of the optimised walks: 4-wide QNodes over every
// object of the scene, one object per leaf (leaf_ref(slot, 1)), boxes from
// conservative world bounds of each object (fast.cu: k_object_boxes) and
// refreshed on the device whenever the instances move.  The ranking of equal
// distances does not depend on this tree: an object's rank comes from the
// reference TLAS leaf that holds it (the metadata's z word).
constexpr uint32_t kEmptyTlas = kLeafBit;  // root of a scene without objects (a leaf of count 0)
constexpr int kTlas4Stack = 40;
// Depth of the BLAS nodes whose boxes bound a mesh for the instance tree: up
// to 2^kSubBoxDepth local boxes per mesh, each corner through the instance
// transform.
constexpr int kSubBoxDepth = 8;

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
    // Instance-level tree.  Per mesh: its local sub-boxes (host_sub, six
    // floats each) at sub_boxes[first .. first + count) and the largest
    // coordinate magnitude they reach.
    struct MeshSub {
        uint32_t first, count;
        float radius;
    };
    std::map<std::tuple<uint32_t, uint32_t, uint32_t, uint32_t>, MeshSub> mesh_sub;
    std::vector<float> host_sub;
    DevBuf<float> sub_boxes;
    DevBuf<QNode> tnodes;         // the tree's nodes (boxes rewritten on every refresh)
    DevBuf<float> tbox;           // float box per tree node (6 floats)
    DevBuf<float> obj_box;        // conservative world box per object (6 floats)
    DevBuf<float> static_box;     // analytic objects' boxes (6 floats per object slot)
    DevBuf<int32_t> tlevels;      // tree nodes by depth, deepest first
    DevBuf<uint32_t> tflag;       // set by the refresh when a box cannot be quantised
    std::vector<int32_t> tlevel_start;
    uint32_t troot = kEmptyTlas, n_tnodes = 0;
    int tlas_stack = 0;
    float static_range = 0.0f;    // largest coordinate magnitude of the analytic objects' boxes
    uint64_t tlas_key = ~0ull, sub_key = ~0ull;
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
    const uint4 *meta;      // x: shape | material << 8, y: instance, z: first slot of its reference TLAS leaf
    const QNode *tnodes;    // instance-level tree
    uint32_t troot;         // its root: a node index, leaf_ref(slot, 1), or kEmptyTlas
};

// The view of a prepared scene; `inst` and `tnodes` may name another copy of
// the per-frame arrays (serving frame sets).
inline FastView fast_view(const FastScene &F, const FastInst *inst = nullptr, const QNode *tnodes = nullptr) {
    return FastView{F.nodes.ptr, F.tris.ptr, inst ? inst : F.inst.ptr, F.obj_meta.ptr, tnodes ? tnodes : F.tnodes.ptr,
                    F.troot};
}

// Rank of an object's candidates (see Best): ~first slot of the reference
// TLAS leaf holding the object, then the slot.
AE_DEV uint64_t object_rank(const uint4 &meta, uint32_t slot) { return (uint64_t(~meta.z) << 32) | slot; }

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

// Sorts child_hits' four (distance, child) pairs nearest first and returns
// how many were hit (misses carry +inf and sort last).
AE_DEV int sort_hits(float tm[4], uint32_t ch[4]) {
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
    return nh;
}

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
    // Next stack entry still no farther than the best hit; false when none.
    auto pop = [&]() {
        while (sp > 0) {
            sp--;
            const uint2 e = sp < SS ? stk[sp * nthreads + tid] : spill[sp - SS];
            if (__uint_as_float(e.y) <= best.t) {
                cur = e.x;
                return true;
            }
        }
        return false;
    };
    for (;;) {
        // Interior nodes until this lane holds a leaf; the warp's lanes then
        // test their leaves' triangles together.
        while (!(cur & kLeafBit)) {
            float tm[4];
            uint32_t ch[4];
            if (T) T->blas++;
            child_hits(V.nodes + cur, lo, inv, tn, best.t, tm, ch);
            const int nh = sort_hits(tm, ch);
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
            } else if (!pop()) {
                return;
            }
        }
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
        if (!pop()) return;
    }
}

// Closest hit of one ray over the whole scene: the instance-level tree
// (nearest child first), analytic objects by the reference intersectors,
// meshes by the 4-wide quantised BLAS.  `stk` is this thread's column of the
// block's shared-memory stack.  T (optional) counts the touches: instance-tree
// nodes, object metadata records, instance records, wide BLAS nodes, triangle
// records.
template <bool WT, int SS = kSharedStack>
AE_DEV Best closest_fast(const DevScene &S, const FastView &V, f3 o, f3 d, float tn, float time, uint2 *stk, int tid,
                         int nt, Touch *T = nullptr) {
    Best best;
    best.t = kFarStart; best.alpha = 0.0f; best.beta = 0.0f;
    best.object = AE_MISS; best.prim = AE_MISS; best.orank = 0; best.lrank = 0;
    if (V.troot == kEmptyTlas) return best;
    const f3 inv = mk(slab_inv(d.x), slab_inv(d.y), slab_inv(d.z));
    uint32_t tstack[kTlas4Stack];
    float tdist[kTlas4Stack];
    int sp = 0;
    uint32_t cur = V.troot;
    // Next stack entry no farther than the best hit; false when none is left.
    auto pop = [&]() {
        while (sp > 0) {
            sp--;
            if (tdist[sp] <= best.t) {
                cur = tstack[sp];
                return true;
            }
        }
        return false;
    };
    for (;;) {
        // Inner nodes until this lane holds an object: the lanes of a warp
        // leave this loop together and then enter their objects together
        // (a lane at a node does not wait through another lane's whole mesh).
        bool live = true;
        while (!(cur & kLeafBit)) {
            float tm[4];
            uint32_t ch[4];
            if (T) T->tlas++;
            child_hits(V.tnodes + cur, o, inv, tn, best.t, tm, ch);
            const int nh = sort_hits(tm, ch);
            if (nh > 0) {
                // prepare_fast checked the tree against kTlas4Stack.
                for (int k = nh - 1; k >= 1; k--) {
                    if (sp < kTlas4Stack) {
                        tstack[sp] = ch[k];
                        tdist[sp] = tm[k];
                        sp++;
                    }
                }
                cur = ch[0];
            } else if (!pop()) {
                live = false;
                break;
            }
        }
        if (!live) break;
        const uint32_t slot = leaf_first(cur);
        const uint4 m = __ldg(V.meta + slot);
        const uint64_t orank = object_rank(m, slot);
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
        if (!pop()) break;
    }
    return best;
}

}  // namespace ae
