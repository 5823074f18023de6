// fast.cu - the optimised closest-hit path.
//
// Data layout (built once per geometry upload, in HBM):
//   * per distinct mesh, a 4-wide BVH collapsed from the reference's binary
//     BLAS (scene/bvh.h).  Collapsing only merges interior nodes, so every
//     leaf - and therefore every triangle slot - is the reference's.  A node
//     is 64 bytes: the node box origin, one power-of-two scale per axis and
//     four child boxes quantised to 8 bits, rounded outward so a decoded box
//     always contains the exact one (no hit can be lost);
//   * triangles in leaf-slot order as 48-byte records {p0, p1, p2}: one
//     contiguous read per leaf instead of an index fetch plus three vertex
//     fetches;
//   * per instance a 48-byte record with the transform and the mesh's node
//     and triangle bases.
//
// Traversal is nearest-child-first with the far children on a shared-memory
// stack that also stores each entry's entry distance, so a popped subtree
// farther than the current hit is skipped without touching its node.
//
// Equal distances: the reference's depth-first walk (hybrid:862-917,
// 617-652) accepts a hit at t == far, so of several hits at the same t the one
// visited LAST wins.  Its walk pops the right child first, and the builder
// gives right subtrees the higher leaf slots, so the visit order is: leaves by
// DESCENDING first slot, primitives within a leaf by ascending slot, objects
// before their triangles.  The kernels rank every candidate by that order and
// keep the highest rank among equal t, which reproduces the reference's answer
// whatever order they visit in.
//
// The triangle test is the reference's HitMeshTriangle (hybrid:564-598) in
// correctly rounded binary32, so t and the barycentrics are bit-identical to
// the plain kernel's; the watertight variant (Woop, Benthin and Wald, "Watertight
// Ray/Triangle Intersection", JCGT 2013) is selected with `quant`.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "context.h"
#include "fast.h"
#include "fast_trace.cuh"
#include "fast_walk.cuh"
#include "kernels.h"
#include "trace_common.cuh"

namespace ae {

// ---------------------------------------------------------------------------
// Host: 4-wide collapse and quantisation
// ---------------------------------------------------------------------------
namespace {

struct Box {
    float lo[3], hi[3];
};
Box node_box(const ae_bvh_node &n) { return Box{{n.min_x, n.min_y, n.min_z}, {n.max_x, n.max_y, n.max_z}}; }
float half_area(const Box &b) {
    const float dx = b.hi[0] - b.lo[0], dy = b.hi[1] - b.lo[1], dz = b.hi[2] - b.lo[2];
    return dx * dy + dy * dz + dz * dx;
}

// Smallest exponent e with (extent / 2^e) <= 255, i.e. 8 bits cover the box.
int axis_exponent(float extent) {
    if (!(extent > 0.0f)) return -126;
    int e = int(std::ceil(std::log2(double(extent) / 255.0)));
    while (std::ldexp(255.0, e) < double(extent)) e++;
    return std::max(e, -126);
}

// Quantise child interval [a, b] in the frame (origin o, scale 2^e) so that
// the decoded interval o + q*2^e, evaluated as the kernel does (fmaf),
// contains it.
void quantise(float o, int e, float a, float b, uint8_t &qa, uint8_t &qb, bool &ok) {
    const float s = std::ldexp(1.0f, e);
    long la = long(std::floor((double(a) - double(o)) / double(s)));
    long lb = long(std::ceil((double(b) - double(o)) / double(s)));
    la = std::max(0L, std::min(255L, la));
    lb = std::max(0L, std::min(255L, lb));
    while (la > 0 && std::fma(float(la), s, o) > a) la--;
    while (lb < 255 && std::fma(float(lb), s, o) < b) lb++;
    ok = ok && std::fma(float(la), s, o) <= a && std::fma(float(lb), s, o) >= b;
    qa = uint8_t(la);
    qb = uint8_t(lb);
}

struct Collapser {
    const ae_bvh_node *bin;  // this mesh's binary nodes
    std::vector<QNode> &out;
    bool ok = true;
    int max_stack = 0;

    // Children of binary node `i` gathered into up to four: repeatedly open
    // the interior child with the largest surface area.
    uint32_t emit(uint32_t i) {
        std::vector<uint32_t> kids = {uint32_t(bin[i].left), uint32_t(bin[i].right)};
        while (kids.size() < 4) {
            int best = -1;
            float area = -1.0f;
            for (size_t k = 0; k < kids.size(); k++) {
                const ae_bvh_node &c = bin[kids[k]];
                if (c.count > 0) continue;
                const float a = half_area(node_box(c));
                if (a > area) { area = a; best = int(k); }
            }
            if (best < 0) break;
            const uint32_t open = kids[best];
            kids.erase(kids.begin() + best);
            kids.insert(kids.begin() + best, uint32_t(bin[open].right));
            kids.insert(kids.begin() + best, uint32_t(bin[open].left));
        }
        const uint32_t self = uint32_t(out.size());
        out.push_back(QNode{});
        QNode q;
        std::memset(&q, 0, sizeof(q));
        Box nb = node_box(bin[i]);
        // Conservative frame: the union of the children.
        Box u = node_box(bin[kids[0]]);
        for (size_t k = 1; k < kids.size(); k++) {
            const Box c = node_box(bin[kids[k]]);
            for (int a = 0; a < 3; a++) { u.lo[a] = std::min(u.lo[a], c.lo[a]); u.hi[a] = std::max(u.hi[a], c.hi[a]); }
        }
        (void)nb;
        q.ox = u.lo[0]; q.oy = u.lo[1]; q.oz = u.lo[2];
        const float org[3] = {q.ox, q.oy, q.oz};
        int ex[3];
        for (int a = 0; a < 3; a++) {
            int e = axis_exponent(u.hi[a] - u.lo[a]);
            // Raise the exponent until the top of the frame is representable.
            for (;;) {
                const float s = std::ldexp(1.0f, e);
                if (std::fma(255.0f, s, org[a]) >= u.hi[a] || e > 127) break;
                e++;
            }
            ex[a] = e;
        }
        q.ex = int8_t(ex[0]); q.ey = int8_t(ex[1]); q.ez = int8_t(ex[2]);
        q.nchild = uint8_t(kids.size());
        for (size_t k = 0; k < kids.size(); k++) {
            const Box c = node_box(bin[kids[k]]);
            for (int a = 0; a < 3; a++) quantise(org[a], ex[a], c.lo[a], c.hi[a], q.lo[a][k], q.hi[a][k], ok);
        }
        for (size_t k = 0; k < kids.size(); k++) {
            const ae_bvh_node &c = bin[kids[k]];
            if (c.count > 0) {
                if (uint32_t(c.count) > kMaxLeafCount || uint32_t(c.left) >= kMaxLeafFirst) ok = false;
                q.child[k] = leaf_ref(uint32_t(c.left) & 0x00ffffffu, uint32_t(c.count) & 0x7fu);
            }
        }
        // Empty slots: an inverted box (lo 255 > hi 0) never hits.
        for (size_t k = kids.size(); k < 4; k++)
            for (int a = 0; a < 3; a++) { q.lo[a][k] = 255; q.hi[a][k] = 0; }
        for (size_t k = 0; k < kids.size(); k++) {
            const ae_bvh_node &c = bin[kids[k]];
            if (c.count <= 0) q.child[k] = emit(kids[k]);
        }
        out[self] = q;
        return self;
    }
};

// Worst-case stack entries of the kernel's loop over this tree: on each
// node the far hit children are pushed (up to nchild - 1).
int stack_need(const std::vector<QNode> &nodes, uint32_t root) {
    const QNode &q = nodes[root];
    int best = 0;
    for (int k = 0; k < q.nchild; k++) {
        if (q.child[k] & kLeafBit) continue;
        best = std::max(best, stack_need(nodes, q.child[k]));
    }
    return (q.nchild - 1) + best;
}

// Boxes of a mesh's binary BLAS nodes at depth kSubBoxDepth (leaves above
// that depth count as they are), appended to `out` as six floats each; they
// cover every triangle of the mesh.  Returns how many.
uint32_t mesh_sub_boxes(const ae_bvh_node *bin, std::vector<float> &out) {
    std::vector<uint32_t> level = {0};
    for (int d = 0; d < kSubBoxDepth; d++) {
        std::vector<uint32_t> next;
        for (uint32_t i : level) {
            if (bin[i].count > 0) next.push_back(i);
            else { next.push_back(uint32_t(bin[i].left)); next.push_back(uint32_t(bin[i].right)); }
        }
        level.swap(next);
    }
    for (uint32_t i : level) {
        const ae_bvh_node &n = bin[i];
        const float b[6] = {n.min_x, n.min_y, n.min_z, n.max_x, n.max_y, n.max_z};
        out.insert(out.end(), b, b + 6);
    }
    return uint32_t(level.size());
}

// World box of a mesh instance from its sub-boxes (double precision; the
// device refresh computes the conservative version of the same bound).
Box instance_box_host(const ae_instance &m, const float *sub, uint32_t count) {
    const double s = (m.scale != 0.0f && m.scale != 1.0f) ? double(m.scale) : 1.0;
    const double qx = m.qx, qy = m.qy, qz = m.qz, qw = m.qw;
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (uint32_t b = 0; b < count; b++) {
        const float *x = sub + 6 * size_t(b);
        for (int k = 0; k < 8; k++) {
            const double v[3] = {(k & 1 ? x[3] : x[0]) * s, (k & 2 ? x[4] : x[1]) * s, (k & 4 ? x[5] : x[2]) * s};
            const double t[3] = {2 * (qy * v[2] - qz * v[1]), 2 * (qz * v[0] - qx * v[2]), 2 * (qx * v[1] - qy * v[0])};
            const double w[3] = {v[0] + qw * t[0] + (qy * t[2] - qz * t[1]) + m.px,
                                 v[1] + qw * t[1] + (qz * t[0] - qx * t[2]) + m.py,
                                 v[2] + qw * t[2] + (qx * t[1] - qy * t[0]) + m.pz};
            for (int a = 0; a < 3; a++) { lo[a] = std::min(lo[a], w[a]); hi[a] = std::max(hi[a], w[a]); }
        }
    }
    Box r;
    for (int a = 0; a < 3; a++) { r.lo[a] = float(lo[a]); r.hi[a] = float(hi[a]); }
    return r;
}

// Binary tree over object boxes with one object per leaf, in ae_bvh_node
// form (a leaf holds its object slot in `left`, count 1): binned SAH over the
// centroids, 16 bins per axis; a median split where the centroids coincide
// or the tree gets deep.
struct ObjectTree {
    const std::vector<Box> &box;
    std::vector<uint32_t> idx;
    std::vector<ae_bvh_node> nodes;

    static float centre(const Box &b, int a) { return 0.5f * (b.lo[a] + b.hi[a]); }

    uint32_t build(uint32_t b, uint32_t e, int depth) {
        const uint32_t self = uint32_t(nodes.size());
        nodes.push_back(ae_bvh_node{});
        Box u = box[idx[b]];
        for (uint32_t i = b + 1; i < e; i++)
            for (int a = 0; a < 3; a++) {
                u.lo[a] = std::min(u.lo[a], box[idx[i]].lo[a]);
                u.hi[a] = std::max(u.hi[a], box[idx[i]].hi[a]);
            }
        ae_bvh_node n;
        std::memset(&n, 0, sizeof(n));
        n.min_x = u.lo[0]; n.min_y = u.lo[1]; n.min_z = u.lo[2];
        n.max_x = u.hi[0]; n.max_y = u.hi[1]; n.max_z = u.hi[2];
        if (e - b == 1) {
            n.left = int32_t(idx[b]);
            n.count = 1;
            nodes[self] = n;
            return self;
        }
        float clo[3] = {1e30f, 1e30f, 1e30f}, chi[3] = {-1e30f, -1e30f, -1e30f};
        for (uint32_t i = b; i < e; i++)
            for (int a = 0; a < 3; a++) {
                clo[a] = std::min(clo[a], centre(box[idx[i]], a));
                chi[a] = std::max(chi[a], centre(box[idx[i]], a));
            }
        constexpr int kBins = 16;
        int axis = -1, split = 0;
        double best = 1e300;
        for (int a = 0; a < 3 && depth < 48; a++) {
            const float ext = chi[a] - clo[a];
            if (!(ext > 0.0f)) continue;
            uint32_t cnt[kBins] = {};
            Box bb[kBins];
            for (int k = 0; k < kBins; k++)
                for (int j = 0; j < 3; j++) { bb[k].lo[j] = 1e30f; bb[k].hi[j] = -1e30f; }
            for (uint32_t i = b; i < e; i++) {
                const Box &x = box[idx[i]];
                const int k = std::min(kBins - 1, int((centre(x, a) - clo[a]) / ext * kBins));
                cnt[k]++;
                for (int j = 0; j < 3; j++) { bb[k].lo[j] = std::min(bb[k].lo[j], x.lo[j]); bb[k].hi[j] = std::max(bb[k].hi[j], x.hi[j]); }
            }
            double right_area[kBins];
            uint32_t right_cnt[kBins];
            Box acc = bb[kBins - 1];
            uint32_t rc = 0;
            for (int k = kBins - 1; k >= 1; k--) {
                if (k < kBins - 1)
                    for (int j = 0; j < 3; j++) { acc.lo[j] = std::min(acc.lo[j], bb[k].lo[j]); acc.hi[j] = std::max(acc.hi[j], bb[k].hi[j]); }
                rc += cnt[k];
                right_area[k] = rc ? half_area(acc) : 0.0;
                right_cnt[k] = rc;
            }
            Box lacc = bb[0];
            uint32_t lc = 0;
            for (int k = 1; k < kBins; k++) {
                if (k > 1)
                    for (int j = 0; j < 3; j++) { lacc.lo[j] = std::min(lacc.lo[j], bb[k - 1].lo[j]); lacc.hi[j] = std::max(lacc.hi[j], bb[k - 1].hi[j]); }
                lc += cnt[k - 1];
                if (!lc || !right_cnt[k]) continue;
                const double cost = double(lc) * half_area(lacc) + double(right_cnt[k]) * right_area[k];
                if (cost < best) { best = cost; axis = a; split = k; }
            }
        }
        uint32_t m = b;
        if (axis >= 0) {
            const float ext = chi[axis] - clo[axis];
            m = uint32_t(std::partition(idx.begin() + b, idx.begin() + e, [&](uint32_t o) {
                            return std::min(kBins - 1, int((centre(box[o], axis) - clo[axis]) / ext * kBins)) < split;
                        }) - idx.begin());
        }
        if (m == b || m == e) {
            int a = 0;
            for (int j = 1; j < 3; j++) if (chi[j] - clo[j] > chi[a] - clo[a]) a = j;
            m = (b + e) / 2;
            std::nth_element(idx.begin() + b, idx.begin() + m, idx.begin() + e,
                             [&](uint32_t x, uint32_t y) { return centre(box[x], a) < centre(box[y], a); });
        }
        const uint32_t l = build(b, m, depth + 1), r = build(m, e, depth + 1);
        n.left = int32_t(l);
        n.right = int32_t(r);
        n.count = 0;
        nodes[self] = n;
        return self;
    }
};

}  // namespace

// The 4-wide quantised BVH of one mesh from its binary BLAS (mesh-relative
// node links, `tri_count` triangles).  Node indices in `out` start at 0; the
// root is returned in `root` (a node index, or a leaf ref for a one-leaf
// mesh).  Checks, before anything reaches a device: every link stays inside
// the tree, every leaf inside the mesh's triangles, every quantised box
// contains its exact box, and the traversal stack bound.
bool build_qbvh(const ae_bvh_node *bin, uint32_t n_bin, uint32_t tri_count, std::vector<QNode> &out, uint32_t &root,
                int &stack, std::string &err) {
    out.clear();
    stack = 0;
    if (n_bin == 0) { err = "empty BLAS"; return false; }
    // The binary tree itself: links in range, acyclic, leaves in range.
    {
        std::vector<uint8_t> seen(n_bin, 0);
        std::vector<uint32_t> todo = {0};
        while (!todo.empty()) {
            const uint32_t i = todo.back();
            todo.pop_back();
            if (i >= n_bin || seen[i]++) { err = "binary BLAS link out of range or repeated"; return false; }
            const ae_bvh_node &n = bin[i];
            if (n.count > 0) {
                if (n.left < 0 || uint64_t(n.left) + uint64_t(n.count) > tri_count) { err = "leaf outside the mesh"; return false; }
                if (uint32_t(n.count) > kMaxLeafCount || uint32_t(n.left) >= kMaxLeafFirst) {
                    err = "leaf beyond the packed reference limits";
                    return false;
                }
            } else {
                if (n.left < 0 || n.right < 0) { err = "negative link"; return false; }
                todo.push_back(uint32_t(n.left));
                todo.push_back(uint32_t(n.right));
            }
        }
    }
    if (bin[0].count > 0) {
        root = leaf_ref(uint32_t(bin[0].left), uint32_t(bin[0].count));
        stack = 0;
        return true;
    }
    Collapser col{bin, out};
    root = col.emit(0);
    if (!col.ok) { err = "a child box cannot be quantised conservatively"; return false; }
    // Final structural check of what the kernel will follow.
    for (size_t i = 0; i < out.size(); i++) {
        const QNode &q = out[i];
        if (q.nchild < 2 || q.nchild > 4) { err = "node child count"; return false; }
        for (int k = 0; k < q.nchild; k++) {
            const uint32_t r = q.child[k];
            if (r & kLeafBit) {
                if (leaf_count(r) == 0 || uint64_t(leaf_first(r)) + leaf_count(r) > tri_count) { err = "leaf ref"; return false; }
            } else if (r >= out.size()) {
                err = "node ref";
                return false;
            }
        }
    }
    stack = stack_need(out, root);
    if (stack + 1 > kFastStack) { err = "tree needs more stack than the kernel holds"; return false; }
    return true;
}

// ---------------------------------------------------------------------------
// Instance-level tree
// ---------------------------------------------------------------------------

// Conservative world box of every object, one warp per object: a mesh
// instance's sub-boxes (its BLAS nodes at depth kSubBoxDepth) with each
// corner through the instance transform in double precision, the extremes
// rounded outward to float; an analytic object's packed box.  Both are
// widened by `margin` on every side, which covers the rounding of the
// kernels' ToLocal and triangle arithmetic for rays that start within the
// scene's coordinate range (the margin is 2^-14 of it).
__global__ void k_object_boxes(const uint4 *__restrict__ meta, const FastInst *__restrict__ inst,
                               const float *__restrict__ sub, const float *__restrict__ static_box, uint32_t n,
                               float margin, float *__restrict__ out) {
    const uint32_t slot = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (slot >= n) return;  // whole warps
    const uint4 m = meta[slot];
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    if ((m.x & 0xff) == AE_SHAPE_MESH) {
        const FastInst I = inst[m.y];
        const double s = (I.scale != 0.0f && I.scale != 1.0f) ? double(I.scale) : 1.0;
        const double qx = I.qx, qy = I.qy, qz = I.qz, qw = I.qw;
        const uint32_t first = I.pad[0], cnt = I.pad[1];
        for (uint32_t j = lane; j < cnt * 8u; j += 32) {
            const float *x = sub + 6 * size_t(first + j / 8);
            const uint32_t k = j & 7u;
            const double v0 = double(k & 1u ? x[3] : x[0]) * s, v1 = double(k & 2u ? x[4] : x[1]) * s,
                         v2 = double(k & 4u ? x[5] : x[2]) * s;
            const double t0 = 2.0 * (qy * v2 - qz * v1), t1 = 2.0 * (qz * v0 - qx * v2), t2 = 2.0 * (qx * v1 - qy * v0);
            const double w[3] = {v0 + qw * t0 + (qy * t2 - qz * t1) + double(I.px),
                                 v1 + qw * t1 + (qz * t0 - qx * t2) + double(I.py),
                                 v2 + qw * t2 + (qx * t1 - qy * t0) + double(I.pz)};
            for (int a = 0; a < 3; a++) { lo[a] = fmin(lo[a], w[a]); hi[a] = fmax(hi[a], w[a]); }
        }
        for (int off = 16; off > 0; off >>= 1)
            for (int a = 0; a < 3; a++) {
                lo[a] = fmin(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], off));
                hi[a] = fmax(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], off));
            }
    } else {
        const float *x = static_box + 6 * size_t(slot);
        for (int a = 0; a < 3; a++) { lo[a] = x[a]; hi[a] = x[3 + a]; }
    }
    if (lane == 0) {
        float *o = out + 6 * size_t(slot);
        for (int a = 0; a < 3; a++) {
            o[a] = __fsub_rd(__double2float_rd(lo[a]), margin);
            o[3 + a] = __fadd_ru(__double2float_ru(hi[a]), margin);
        }
    }
}

// Smallest power-of-two scale whose 255 steps from `org` reach `top`
// (the host collapser's frame rule); false when none fits the exponent range.
__device__ bool frame_exponent(float org, float top, int &e) {
    const float extent = top - org;
    e = -126;
    if (extent > 0.0f) {
        e = int(ceil(log2(double(extent) / 255.0)));
        while (ldexp(255.0, e) < double(extent)) e++;
        e = max(e, -126);
    }
    while (e <= 127 && fmaf(255.0f, ldexpf(1.0f, e), org) < top) e++;
    return e <= 127;
}

// Child interval [a, b] quantised outward in the frame (org, 2^e): the
// decoded bounds org + q 2^e (fmaf) contain it.
__device__ bool quantise_outward(float org, int e, float a, float b, uint8_t &qa, uint8_t &qb) {
    const float sc = ldexpf(1.0f, e);
    double la = floor((double(a) - double(org)) / double(sc)), lb = ceil((double(b) - double(org)) / double(sc));
    la = fmin(fmax(la, 0.0), 255.0);
    lb = fmin(fmax(lb, 0.0), 255.0);
    int ia = int(la), ib = int(lb);
    while (ia > 0 && fmaf(float(ia), sc, org) > a) ia--;
    while (ib < 255 && fmaf(float(ib), sc, org) < b) ib++;
    qa = uint8_t(ia);
    qb = uint8_t(ib);
    return fmaf(float(ia), sc, org) <= a && fmaf(float(ib), sc, org) >= b;
}

// One level of the instance tree's bottom-up refresh (levels deepest first):
// a node's float box is the union of its children's (objects' boxes for leaf
// children), and its children are re-quantised in the node's new frame.  A
// child whose box is empty or not finite becomes an unused slot.  Sets *bad
// when a box cannot be quantised conservatively.
__global__ void k_instance_tree_level(QNode *__restrict__ nodes, float *__restrict__ nbox,
                                      const float *__restrict__ obj_box, const int32_t *__restrict__ level,
                                      int32_t count, uint32_t *bad) {
    const int32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const int32_t ni = level[k];
    QNode q = nodes[ni];
    float cb[4][6];
    bool cv[4];
    float u[6] = {3.402823466e38f, 3.402823466e38f, 3.402823466e38f, -3.402823466e38f, -3.402823466e38f,
                  -3.402823466e38f};
    bool any = false;
    for (int c = 0; c < 4; c++) {
        cv[c] = false;
        if (c >= q.nchild) continue;
        const uint32_t ref = q.child[c];
        const float *x = (ref & kLeafBit) ? obj_box + 6 * size_t(leaf_first(ref)) : nbox + 6 * size_t(ref);
        bool ok = true;
        for (int a = 0; a < 6; a++) { cb[c][a] = x[a]; ok = ok && isfinite(x[a]); }
        for (int a = 0; a < 3; a++) ok = ok && cb[c][a] <= cb[c][3 + a];
        cv[c] = ok;
        if (!ok) continue;
        any = true;
        for (int a = 0; a < 3; a++) { u[a] = fminf(u[a], cb[c][a]); u[3 + a] = fmaxf(u[3 + a], cb[c][3 + a]); }
    }
    bool good = true;
    int ex[3] = {0, 0, 0};
    if (any) {
        q.ox = u[0]; q.oy = u[1]; q.oz = u[2];
        for (int a = 0; a < 3; a++) good = frame_exponent(u[a], u[3 + a], ex[a]) && good;
    } else {
        q.ox = q.oy = q.oz = 0.0f;
        u[0] = u[1] = u[2] = __int_as_float(0x7f800000);
        u[3] = u[4] = u[5] = -__int_as_float(0x7f800000);
    }
    q.ex = int8_t(good ? ex[0] : 0); q.ey = int8_t(good ? ex[1] : 0); q.ez = int8_t(good ? ex[2] : 0);
    const float org[3] = {q.ox, q.oy, q.oz};
    for (int c = 0; c < 4; c++) {
        if (cv[c] && any && good) {
            for (int a = 0; a < 3; a++)
                good = quantise_outward(org[a], ex[a], cb[c][a], cb[c][3 + a], q.lo[a][c], q.hi[a][c]) && good;
        } else {
            for (int a = 0; a < 3; a++) { q.lo[a][c] = 255; q.hi[a][c] = 0; }
        }
    }
    if (!good) atomicExch(bad, 1u);
    nodes[ni] = q;
    float *o = nbox + 6 * size_t(ni);
    for (int a = 0; a < 6; a++) o[a] = u[a];
}

// Topology of the instance-level tree for the current objects (host, per
// scene layout): an object tree over host bounds, collapsed 4-wide by the
// BLAS collapser.  The boxes uploaded here are replaced by the device
// refresh.
static int build_instance_tree(Ctx *c, FastScene &F) {
    const uint32_t n = c->n_objects;
    F.n_tnodes = 0;
    F.tlas_stack = 0;
    F.troot = kEmptyTlas;
    F.static_range = 0.0f;
    if (n == 0) return AE_OK;
    if (n >= kMaxLeafFirst) return c->fail(AE_ERR_LAYOUT, "%u objects: the instance tree addresses at most %u", n, kMaxLeafFirst);
    std::vector<Box> boxes(n);
    std::vector<float> stat(size_t(n) * 6, 0.0f);
    for (uint32_t s = 0; s < n; s++) {
        const ae_object &o = c->host_objects[s];
        if (o.shapeType == AE_SHAPE_MESH) {
            const ae_instance &m = c->host_instances[o.instanceIndex];
            const FastScene::MeshSub &ms = F.mesh_sub.at(std::make_tuple(m.vertexBase, m.indexBase, m.triangleCount, m.blasBase));
            boxes[s] = instance_box_host(m, F.host_sub.data() + 6 * size_t(ms.first), ms.count);
        } else {
            const ae_aabb b = analytic_box(o);
            boxes[s] = Box{{b.min_x, b.min_y, b.min_z}, {b.max_x, b.max_y, b.max_z}};
            std::memcpy(&stat[6 * size_t(s)], &b, 24);
            for (int a = 0; a < 3; a++)
                F.static_range = std::max(F.static_range, std::max(std::fabs(boxes[s].lo[a]), std::fabs(boxes[s].hi[a])));
        }
    }
    ObjectTree T{boxes, {}, {}};
    T.idx.resize(n);
    for (uint32_t s = 0; s < n; s++) T.idx[s] = s;
    T.nodes.reserve(2 * size_t(n));
    T.build(0, n, 0);
    std::vector<QNode> out;
    uint32_t root;
    if (T.nodes[0].count > 0) {
        root = leaf_ref(uint32_t(T.nodes[0].left), 1);
    } else {
        Collapser col{T.nodes.data(), out};
        root = col.emit(0);
        F.tlas_stack = stack_need(out, root);
        if (F.tlas_stack > kTlas4Stack)
            return c->fail(AE_ERR_LAYOUT, "instance tree needs %d stack entries (> %d)", F.tlas_stack, kTlas4Stack);
    }
    // Nodes by depth, deepest first, for the bottom-up refresh.
    std::vector<int32_t> depth(out.size(), 0), order;
    int maxd = 0;
    for (size_t i = 0; i < out.size(); i++)
        for (int k = 0; k < out[i].nchild; k++)
            if (!(out[i].child[k] & kLeafBit)) {
                depth[out[i].child[k]] = depth[i] + 1;
                maxd = std::max(maxd, depth[i] + 1);
            }
    F.tlevel_start.assign(1, 0);
    for (int d = maxd; d >= 0 && !out.empty(); d--) {
        for (size_t i = 0; i < out.size(); i++)
            if (depth[i] == d) order.push_back(int32_t(i));
        F.tlevel_start.push_back(int32_t(order.size()));
    }
    const size_t nn = std::max<size_t>(out.size(), 1);
    if (F.tnodes.reserve(nn) || F.tbox.reserve(nn * 6) || F.tlevels.reserve(std::max<size_t>(order.size(), 1)) ||
        F.obj_box.reserve(size_t(n) * 6) || F.static_box.reserve(size_t(n) * 6) || F.tflag.reserve(1))
        return c->fail(AE_ERR_OOM, "instance tree");
    int rc;
    if (!out.empty() &&
        ((rc = c->cuda(cudaMemcpyAsync(F.tnodes.ptr, out.data(), out.size() * sizeof(QNode), cudaMemcpyHostToDevice,
                                       c->stream), "upload instance tree")) ||
         (rc = c->cuda(cudaMemcpyAsync(F.tlevels.ptr, order.data(), order.size() * sizeof(int32_t),
                                       cudaMemcpyHostToDevice, c->stream), "upload instance tree levels"))))
        return rc;
    if ((rc = c->cuda(cudaMemcpyAsync(F.static_box.ptr, stat.data(), stat.size() * sizeof(float), cudaMemcpyHostToDevice,
                                      c->stream), "upload object boxes")))
        return rc;
    // The host copies must outlive the asynchronous copies.
    if ((rc = c->cuda(cudaStreamSynchronize(c->stream), "instance tree"))) return rc;
    F.n_tnodes = uint32_t(out.size());
    F.troot = root;
    return AE_OK;
}

// Device refresh of the instance tree's boxes from the current instance
// records (after every upload or refit).
static int refresh_instance_tree(Ctx *c, FastScene &F) {
    if (F.n_tnodes == 0) return AE_OK;
    // Coordinate range of the scene for the margin of the object boxes.
    float range = 1.0f;
    for (uint32_t s = 0; s < c->n_objects; s++) {
        const ae_object &o = c->host_objects[s];
        if (o.shapeType == AE_SHAPE_MESH) {
            const ae_instance &m = c->host_instances[o.instanceIndex];
            const FastScene::MeshSub &ms = F.mesh_sub.at(std::make_tuple(m.vertexBase, m.indexBase, m.triangleCount, m.blasBase));
            const float sc = (m.scale != 0.0f && m.scale != 1.0f) ? std::fabs(m.scale) : 1.0f;
            const float r = std::max(std::fabs(m.px), std::max(std::fabs(m.py), std::fabs(m.pz))) + 1.75f * sc * ms.radius;
            range = std::max(range, r);
        }
    }
    range = std::max(range, F.static_range);
    const float margin = std::ldexp(range, -14);
    const uint32_t n = c->n_objects;
    int rc;
    if ((rc = c->cuda(cudaMemsetAsync(F.tflag.ptr, 0, sizeof(uint32_t), c->stream), "instance tree flag"))) return rc;
    k_object_boxes<<<(n * 32 + 255) / 256, 256, 0, c->stream>>>(F.obj_meta.ptr, F.inst.ptr, F.sub_boxes.ptr,
                                                                 F.static_box.ptr, n, margin, F.obj_box.ptr);
    for (size_t l = 0; l + 1 < F.tlevel_start.size(); l++) {
        const int32_t cnt = F.tlevel_start[l + 1] - F.tlevel_start[l];
        if (cnt <= 0) continue;
        k_instance_tree_level<<<(cnt + 127) / 128, 128, 0, c->stream>>>(F.tnodes.ptr, F.tbox.ptr, F.obj_box.ptr,
                                                                       F.tlevels.ptr + F.tlevel_start[l], cnt, F.tflag.ptr);
    }
    return c->cuda(cudaGetLastError(), "instance tree refresh");
}

int prepare_fast(Ctx *c) {
    // Not ready until this call accepts the current scene: every early
    // return below leaves the optimised structures unusable.
    c->fast_ready = false;
    if (!c->geometry_uploaded || !c->scene_uploaded) return c->fail(AE_ERR_STATE, "prepare before uploads");
    if (!c->fast) c->fast = new (std::nothrow) FastScene();
    if (!c->fast) return c->fail(AE_ERR_OOM, "fast scene");
    FastScene &F = *c->fast;
    if (F.geometry_key != c->geometry_version) {
        // New geometry arrays: every mesh is converted again (the device
        // buffers are reused).
        F.mesh_roots.clear();
        F.host_nodes.clear();
        F.host_tris.clear();
        F.mesh_sub.clear();
        F.host_sub.clear();
        F.max_stack = 0;
        F.shade16_tris = 0;
        F.geometry_key = c->geometry_version;
        F.geometry_dirty = true;
    }
    // Geometry-derived part: rebuilt when new meshes appear.
    bool rebuilt = false;
    for (uint32_t i = 0; i < c->n_instances; i++) {
        const ae_instance &m = c->host_instances[i];
        const auto key = std::make_tuple(m.vertexBase, m.indexBase, m.triangleCount, m.blasBase);
        if (F.mesh_roots.count(key)) continue;
        // Triangle records of this mesh in slot order.
        const uint32_t tri_base = uint32_t(F.host_tris.size() / 12);
        F.host_tris.resize(F.host_tris.size() + size_t(m.triangleCount) * 12);
        float *dst = F.host_tris.data() + size_t(tri_base) * 12;
        for (uint32_t t = 0; t < m.triangleCount; t++) {
            for (int v = 0; v < 3; v++) {
                const ae_vertex &vx = c->host_vertices[m.vertexBase + c->host_indices[m.indexBase + 3 * t + v]];
                dst[12 * t + 3 * v + 0] = vx.px;
                dst[12 * t + 3 * v + 1] = vx.py;
                dst[12 * t + 3 * v + 2] = vx.pz;
            }
            dst[12 * t + 9] = dst[12 * t + 10] = dst[12 * t + 11] = 0.0f;
        }
        uint32_t root;
        std::vector<QNode> local;
        int need = 0;
        std::string err;
        if (!build_qbvh(c->host_blas.data() + m.blasBase, uint32_t(c->n_blas - m.blasBase), m.triangleCount, local,
                        root, need, err))
            return c->fail(AE_ERR_LAYOUT, "4-wide BVH of instance %u: %s", i, err.c_str());
        const uint32_t before = uint32_t(F.host_nodes.size());
        for (QNode &q : local)
            for (int k = 0; k < q.nchild; k++)
                if (!(q.child[k] & kLeafBit)) q.child[k] += before;
        if (!(root & kLeafBit)) root += before;
        F.host_nodes.insert(F.host_nodes.end(), local.begin(), local.end());
        F.max_stack = std::max(F.max_stack, need);
        F.mesh_roots[key] = std::make_pair(root, tri_base);
        FastScene::MeshSub ms;
        ms.first = uint32_t(F.host_sub.size() / 6);
        ms.count = mesh_sub_boxes(c->host_blas.data() + m.blasBase, F.host_sub);
        ms.radius = 0.0f;
        for (size_t k = size_t(ms.first) * 6; k < F.host_sub.size(); k++) ms.radius = std::max(ms.radius, std::fabs(F.host_sub[k]));
        F.mesh_sub[key] = ms;
        F.geometry_dirty = true;
    }
    if (F.max_stack + 1 > kFastStack)
        return c->fail(AE_ERR_LAYOUT, "4-wide BVH needs %d stack entries (> %d)", F.max_stack + 1, kFastStack);
    int rc;
    if (F.geometry_dirty) {
        rebuilt = true;
        F.n_nodes = uint32_t(F.host_nodes.size());
        F.n_tris = uint32_t(F.host_tris.size() / 12);
        if (F.nodes.reserve(std::max<size_t>(F.n_nodes, 1)) || F.tris.reserve(std::max<size_t>(size_t(F.n_tris) * 3, 1)))
            return c->fail(AE_ERR_OOM, "fast scene buffers");
        if (F.n_nodes && (rc = c->cuda(cudaMemcpyAsync(F.nodes.ptr, F.host_nodes.data(), F.n_nodes * sizeof(QNode),
                                                       cudaMemcpyHostToDevice, c->stream), "upload nodes")))
            return rc;
        if ((rc = c->cuda(cudaMemcpyAsync(F.tris.ptr, F.host_tris.data(), F.host_tris.size() * sizeof(float),
                                          cudaMemcpyHostToDevice, c->stream), "upload triangles")))
            return rc;
        if (F.sub_boxes.reserve(std::max<size_t>(F.host_sub.size(), 1))) return c->fail(AE_ERR_OOM, "mesh sub-boxes");
        if (!F.host_sub.empty() &&
            (rc = c->cuda(cudaMemcpyAsync(F.sub_boxes.ptr, F.host_sub.data(), F.host_sub.size() * sizeof(float),
                                          cudaMemcpyHostToDevice, c->stream), "upload mesh sub-boxes")))
            return rc;
        F.geometry_dirty = false;
    }
    // Scene-derived part: instances and object metadata, per upload.
    if (F.scene_key != c->scene_version || rebuilt) {
        std::vector<FastInst> fi(std::max<uint32_t>(c->n_instances, 1));
        for (uint32_t i = 0; i < c->n_instances; i++) {
            const ae_instance &m = c->host_instances[i];
            const auto &rt = F.mesh_roots[std::make_tuple(m.vertexBase, m.indexBase, m.triangleCount, m.blasBase)];
            FastInst &f = fi[i];
            f.px = m.px; f.py = m.py; f.pz = m.pz; f.scale = m.scale;
            f.qx = m.qx; f.qy = m.qy; f.qz = m.qz; f.qw = m.qw;
            f.root = rt.first;
            f.tri_base = rt.second;
            const FastScene::MeshSub &ms = F.mesh_sub.at(std::make_tuple(m.vertexBase, m.indexBase, m.triangleCount, m.blasBase));
            f.pad[0] = ms.first;
            f.pad[1] = ms.count;
        }
        // Each object's rank comes from the reference TLAS leaf that holds it.
        std::vector<uint32_t> leaf_first_of(std::max<uint32_t>(c->n_objects, 1), 0u);
        for (const ae_bvh_node &nd : c->host_tlas)
            if (nd.count > 0)
                for (int32_t k = 0; k < nd.count; k++)
                    if (uint32_t(nd.left + k) < c->n_objects) leaf_first_of[nd.left + k] = uint32_t(nd.left);
        std::vector<uint4> meta(std::max<uint32_t>(c->n_objects, 1));
        F.has_volumes = false;
        for (uint32_t s = 0; s < c->n_objects; s++) {
            const ae_object &o = c->host_objects[s];
            meta[s] = make_uint4(o.shapeType | (o.colorType << 8), o.instanceIndex, leaf_first_of[s], 0u);
            if (o.colorType == AE_MAT_ISOTROPIC) F.has_volumes = true;
        }
        if (F.inst.reserve(fi.size()) || F.obj_meta.reserve(meta.size())) return c->fail(AE_ERR_OOM, "fast scene");
        if ((rc = c->cuda(cudaMemcpyAsync(F.inst.ptr, fi.data(), fi.size() * sizeof(FastInst), cudaMemcpyHostToDevice,
                                          c->stream), "upload instances")))
            return rc;
        if ((rc = c->cuda(cudaMemcpyAsync(F.obj_meta.ptr, meta.data(), meta.size() * sizeof(uint4),
                                          cudaMemcpyHostToDevice, c->stream), "upload metadata")))
            return rc;
        if (F.tlas_key != c->scene_version_layout || F.sub_key != c->geometry_version) {
            F.tlas_key = ~0ull;
            if ((rc = build_instance_tree(c, F))) return rc;
            F.tlas_key = c->scene_version_layout;
            F.sub_key = c->geometry_version;
        }
        if ((rc = refresh_instance_tree(c, F))) return rc;
        if ((rc = c->cuda(cudaStreamSynchronize(c->stream), "prepare fast"))) return rc;
        if (F.n_tnodes) {
            uint32_t bad = 0;
            if ((rc = c->cuda(cudaMemcpy(&bad, F.tflag.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost), "instance tree flag")))
                return rc;
            if (bad) return c->fail(AE_ERR_LAYOUT, "instance tree: an object box cannot be quantised conservatively");
        }
        F.scene_key = c->scene_version;
    }
    if (F.has_volumes)
        return c->fail(AE_ERR_STATE, "participating media consume RNG in the reference's visit order; use the plain kernel");
    c->fast_ready = true;
    return AE_OK;
}

// The precision form's shading records: per triangle, in the optimised
// BVH's slot order, the three vertex normals and UVs rounded to FP16
// (round to nearest even), 32 bytes (layout in wf_common.cuh).
int prepare_precision(Ctx *c) {
    int rc = prepare_fast(c);
    if (rc) return rc;
    FastScene &F = *c->fast;
    if (F.shade16_tris == F.n_tris && F.shade16.ptr) return AE_OK;
    std::vector<uint16_t> h(size_t(std::max(F.n_tris, 1u)) * 16, 0);
    auto half_bits = [](float x) {
        const __half v = __float2half_rn(x);
        uint16_t b;
        std::memcpy(&b, &v, 2);
        return b;
    };
    for (const auto &kv : F.mesh_roots) {
        const uint32_t vbase = std::get<0>(kv.first), ibase = std::get<1>(kv.first), tris = std::get<2>(kv.first);
        const uint32_t tri_base = kv.second.second;
        for (uint32_t t = 0; t < tris; t++) {
            uint16_t *r = h.data() + (size_t(tri_base) + t) * 16;
            for (int v = 0; v < 3; v++) {
                const ae_vertex &vx = c->host_vertices[vbase + c->host_indices[ibase + 3 * t + v]];
                r[3 * v + 0] = half_bits(vx.nx);
                r[3 * v + 1] = half_bits(vx.ny);
                r[3 * v + 2] = half_bits(vx.nz);
                r[9 + 2 * v] = half_bits(vx.u);
                r[10 + 2 * v] = half_bits(vx.v);
            }
        }
    }
    if (F.shade16.reserve(size_t(std::max(F.n_tris, 1u)) * 2)) return c->fail(AE_ERR_OOM, "FP16 shading records");
    if ((rc = c->cuda(cudaMemcpyAsync(F.shade16.ptr, h.data(), h.size() * 2, cudaMemcpyHostToDevice, c->stream),
                      "upload FP16 shading records")))
        return rc;
    if ((rc = c->cuda(cudaStreamSynchronize(c->stream), "FP16 shading records"))) return rc;
    F.shade16_tris = F.n_tris;
    return AE_OK;
}

void destroy_fast(Ctx *c) {
    delete c->fast;
    c->fast = nullptr;
}

// Closest hit over a ray batch; one thread per ray.  The occupancy bound
// (8 blocks of 128 per SM, so at most 64 registers) was chosen by timing on
// the B200: 12 % more rays/s than the unbounded 79-register build, whose
// 6 resident blocks left the latency-bound walk short of warps.
template <bool WT>
__global__ void __launch_bounds__(128, 8) k_closest_fast(DevScene S, FastView V, const ae_ray *__restrict__ rays,
                                                      uint32_t n, ae_hit *__restrict__ hits) {
    extern __shared__ uint2 stk[];
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 *rp = reinterpret_cast<const float4 *>(rays + i);
    const float4 r0 = __ldg(rp), r1 = __ldg(rp + 1);
    const Best best = closest_fast<WT>(S, V, mk(r0.x, r0.y, r0.z), mk(r1.x, r1.y, r1.z), r0.w, r1.w, stk,
                                       threadIdx.x, blockDim.x);
    const bool any = best.object != AE_MISS;
    ae_hit out;
    out.t = any ? best.t : 0.0f;
    out.alpha = any ? best.alpha : 0.0f;
    out.beta = any ? best.beta : 0.0f;
    out.object = best.object;
    out.prim = best.prim;
    hits[i] = out;
}

// The optimised walk with its touches counted (outside timed regions): per
// ray set, TLAS nodes, object metadata records, instance records, wide BLAS
// nodes and triangle records fetched, summed in 64-bit.
template <bool WT>
__global__ void __launch_bounds__(128) k_count_fast(DevScene S, FastView V, const ae_ray *__restrict__ rays,
                                                    uint32_t n, unsigned long long *__restrict__ totals) {
    extern __shared__ uint2 stk[];
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    Touch T = {0, 0, 0, 0, 0, 0, 0};
    if (i < n) {
        const float4 *rp = reinterpret_cast<const float4 *>(rays + i);
        const float4 r0 = __ldg(rp), r1 = __ldg(rp + 1);
        const Best best = closest_fast<WT>(S, V, mk(r0.x, r0.y, r0.z), mk(r1.x, r1.y, r1.z), r0.w, r1.w, stk,
                                           threadIdx.x, blockDim.x, &T);
        T.winners = best.object != AE_MISS ? 1u : 0u;
    }
    const uint32_t v[6] = {T.tlas, T.objects, T.instances, T.blas, T.tris, T.winners};
    for (int k = 0; k < 6; k++) {
        unsigned long long x = v[k];
        for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
        if ((threadIdx.x & 31) == 0 && x) atomicAdd(totals + k, x);
    }
}

// The same closest hit on the step-wise Walker, for incoherent ray sets
// (bounce rays): a persistent grid where each lane starts its next ray as soon
// as one finishes.  Bit-identical hits.
//
// DYN: rays are handed out in chunks of kWalkChunk consecutive rays per warp
// from a global counter, and the lanes of a warp take theirs from the warp's
// current chunk, so the rays a warp has in flight stay close in the input
// order (neighbouring pixels: neighbouring origins and nodes).  On a
// 1.3M-ray bounce set this took 3.70 -> 3.31 ms; on the current walker, runs
// of 32 rays beat 64 and 128 (1.72 / 1.76 / 1.96 ms).  It keeps every block busy
// to the end of the launch, which suits a launch that has the GPU to itself;
// the smaller launches of the pipelined host-buffer call, which overlap on
// three streams, use the static assignment (lane i: rays i, i + grid size,
// ...), whose blocks retire early and make room for the next launch.
constexpr uint32_t kWalkChunk = 32;
constexpr uint32_t kWalkDynamicMin = (1u << 19) + 1;  // above the host pipeline's largest chunk

template <bool DYN>
__global__ void __launch_bounds__(128, kWalkBlocksPerSm) k_closest_walk(DevScene S, FastView V,
                                                                     const ae_ray *__restrict__ rays, uint32_t n,
                                                                     ae_hit *__restrict__ hits, uint32_t *next) {
    extern __shared__ uint2 stk[];
    if (!DYN) {
        const uint32_t stride = gridDim.x * blockDim.x;
        uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
        Walker<false> w;
        WalkStacks<> K;
        bool active = k < n;
        if (active) {
            const ae_ray r = rays[k];
            w.start(V, mk(r.ox, r.oy, r.oz), mk(r.dx, r.dy, r.dz), r.tnear, r.time);
        }
        uint32_t iter = 0;
        for (;;) {
            const uint32_t am = __ballot_sync(0xffffffffu, active);
            if (!am) break;
            // Only the warp's largest phase group steps (warp_pick_group).
            const uint32_t pick = warp_pick_group(active ? w.group() : 0u, active, am, iter);
            if (!active || w.group() != pick || !w.step(S, V, K, stk, threadIdx.x, blockDim.x)) continue;
            const Best &b = w.best;
            const bool any = b.object != AE_MISS;
            ae_hit h;
            h.t = any ? b.t : 0.0f;
            h.alpha = any ? b.alpha : 0.0f;
            h.beta = any ? b.beta : 0.0f;
            h.object = b.object;
            h.prim = b.prim;
            hits[k] = h;
            k += stride;
            active = k < n;
            if (active) {
                const ae_ray r = rays[k];
                w.start(V, mk(r.ox, r.oy, r.oz), mk(r.dx, r.dy, r.dz), r.tnear, r.time);
            }
        }
        return;
    }
    const uint32_t lane = threadIdx.x & 31, below = (1u << lane) - 1u;
    Walker<false> w;
    WalkStacks<> K;
    uint32_t k = 0, cbase = 0, cend = 0;  // cbase/cend: the warp's chunk, the same in every lane
    uint32_t iter = 0;
    bool active = false, need = true, exhausted = false;
    for (;;) {
        // Lanes without a ray take the next ones of the warp's chunk, in lane
        // order; a new chunk is fetched when it runs out.
        uint32_t m = __ballot_sync(0xffffffffu, need);
        while (m && !exhausted) {
            if (cbase >= cend) {
                uint32_t b = 0;
                if (lane == 0) b = atomicAdd(next, kWalkChunk);
                b = __shfl_sync(0xffffffffu, b, 0);
                if (b >= n) {
                    exhausted = true;
                    break;
                }
                cbase = b;
                cend = min(b + kWalkChunk, n);
            }
            const uint32_t take = min(cend - cbase, uint32_t(__popc(m)));
            if (need && uint32_t(__popc(m & below)) < take) {
                k = cbase + __popc(m & below);
                need = false;
                active = true;
                const ae_ray r = rays[k];
                w.start(V, mk(r.ox, r.oy, r.oz), mk(r.dx, r.dy, r.dz), r.tnear, r.time);
            }
            cbase += take;
            m = __ballot_sync(0xffffffffu, need);
        }
        const uint32_t am = __ballot_sync(0xffffffffu, active);
        if (!am) break;
        // Only the warp's largest phase group steps (warp_pick_group): on the
        // 1080p bounce set 3.31 -> 2.70 ms.
        const uint32_t pick = warp_pick_group(w.group(), active, am, iter);
        if (active && w.group() == pick && w.step(S, V, K, stk, threadIdx.x, blockDim.x)) {
            const Best &b = w.best;
            const bool any = b.object != AE_MISS;
            ae_hit h;
            h.t = any ? b.t : 0.0f;
            h.alpha = any ? b.alpha : 0.0f;
            h.beta = any ? b.beta : 0.0f;
            h.object = b.object;
            h.prim = b.prim;
            hits[k] = h;
            active = false;
            need = true;
        }
    }
}

cudaError_t launch_closest_walk(Ctx *c, const ae_ray *rays, uint32_t n, ae_hit *hits, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    FastScene &F = *c->fast;
    FastView V = fast_view(F);
    const int threads = 128;
    const size_t smem = size_t(kSharedStack) * threads * sizeof(uint2);
    static int per_sm = 0, sms = 0;
    if (!per_sm) {
        cudaFuncSetAttribute(k_closest_walk<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        cudaFuncSetAttribute(k_closest_walk<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_closest_walk<true>, threads, smem);
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        per_sm = std::max(per_sm, 1);
    }
    const uint32_t grid = std::min<uint32_t>(uint32_t(per_sm) * uint32_t(sms), (n + threads - 1) / threads);
    if (n < kWalkDynamicMin) {
        k_closest_walk<false><<<grid, threads, smem, st>>>(c->scene(), V, rays, n, hits, nullptr);
        return cudaGetLastError();
    }
    if (F.walk_next.reserve(FastScene::kWalkCounters)) return cudaErrorMemoryAllocation;
    uint32_t *next = F.walk_next.ptr + (F.walk_pos++ % FastScene::kWalkCounters);
    cudaError_t e = cudaMemsetAsync(next, 0, sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    k_closest_walk<true><<<grid, threads, smem, st>>>(c->scene(), V, rays, n, hits, next);
    return cudaGetLastError();
}

cudaError_t launch_count_fast(Ctx *c, const ae_ray *rays, uint32_t n, bool quant, unsigned long long *totals,
                              cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    FastScene &F = *c->fast;
    FastView V = fast_view(F);
    const int threads = 128;
    const size_t smem = size_t(kSharedStack) * threads * sizeof(uint2);
    if (quant) {
        cudaFuncSetAttribute(k_count_fast<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        k_count_fast<true><<<(n + threads - 1) / threads, threads, smem, st>>>(c->scene(), V, rays, n, totals);
    } else {
        cudaFuncSetAttribute(k_count_fast<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        k_count_fast<false><<<(n + threads - 1) / threads, threads, smem, st>>>(c->scene(), V, rays, n, totals);
    }
    return cudaGetLastError();
}

cudaError_t launch_closest_fast(Ctx *c, const ae_ray *rays, uint32_t n, ae_hit *hits, bool quant, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    FastScene &F = *c->fast;
    FastView V = fast_view(F);
    const int threads = 128;
    const size_t smem = size_t(kSharedStack) * threads * sizeof(uint2);
    if (quant) {
        cudaFuncSetAttribute(k_closest_fast<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        k_closest_fast<true><<<(n + threads - 1) / threads, threads, smem, st>>>(c->scene(), V, rays, n, hits);
    } else {
        cudaFuncSetAttribute(k_closest_fast<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        k_closest_fast<false><<<(n + threads - 1) / threads, threads, smem, st>>>(c->scene(), V, rays, n, hits);
    }
    return cudaGetLastError();
}

}  // namespace ae

extern "C" int ae_build_wide_bvh(const ae_bvh_node *blas, uint32_t n_nodes, uint32_t tri_count, void *out_nodes,
                                 uint32_t capacity, uint32_t *out_count, uint32_t *out_root, int32_t *out_stack) {
    if (!blas || !out_count || !out_root || !out_stack) return AE_ERR_INVALID;
    std::vector<ae::QNode> nodes;
    uint32_t root = 0;
    int stack = 0;
    std::string err;
    if (!ae::build_qbvh(blas, n_nodes, tri_count, nodes, root, stack, err)) {
        fprintf(stderr, "ae_build_wide_bvh: %s\n", err.c_str());
        return AE_ERR_LAYOUT;
    }
    *out_count = uint32_t(nodes.size());
    *out_root = root;
    *out_stack = stack;
    if (nodes.size() > capacity || (!out_nodes && !nodes.empty())) return AE_ERR_OVERSIZE;
    if (!nodes.empty()) std::memcpy(out_nodes, nodes.data(), nodes.size() * sizeof(ae::QNode));
    return AE_OK;
}
