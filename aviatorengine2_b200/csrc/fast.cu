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
#include "kernels.h"
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
    uint32_t n_nodes = 0, n_tris = 0;
    int max_stack = 0;
    uint64_t geometry_key = 0, scene_key = ~0ull;
    bool has_volumes = false;
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

int prepare_fast(Ctx *c) {
    if (!c->geometry_uploaded || !c->scene_uploaded) return c->fail(AE_ERR_STATE, "prepare before uploads");
    if (!c->fast) c->fast = new (std::nothrow) FastScene();
    if (!c->fast) return c->fail(AE_ERR_OOM, "fast scene");
    FastScene &F = *c->fast;
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
        rebuilt = true;
    }
    if (F.max_stack + 1 > kFastStack)
        return c->fail(AE_ERR_LAYOUT, "4-wide BVH needs %d stack entries (> %d)", F.max_stack + 1, kFastStack);
    int rc;
    if (rebuilt) {
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
            f.pad[0] = f.pad[1] = 0;
        }
        std::vector<uint4> meta(std::max<uint32_t>(c->n_objects, 1));
        F.has_volumes = false;
        for (uint32_t s = 0; s < c->n_objects; s++) {
            const ae_object &o = c->host_objects[s];
            meta[s] = make_uint4(o.shapeType | (o.colorType << 8), o.instanceIndex, 0u, 0u);
            if (o.colorType == AE_MAT_ISOTROPIC) F.has_volumes = true;
        }
        if (F.inst.reserve(fi.size()) || F.obj_meta.reserve(meta.size())) return c->fail(AE_ERR_OOM, "fast scene");
        if ((rc = c->cuda(cudaMemcpyAsync(F.inst.ptr, fi.data(), fi.size() * sizeof(FastInst), cudaMemcpyHostToDevice,
                                          c->stream), "upload instances")))
            return rc;
        if ((rc = c->cuda(cudaMemcpyAsync(F.obj_meta.ptr, meta.data(), meta.size() * sizeof(uint4),
                                          cudaMemcpyHostToDevice, c->stream), "upload metadata")))
            return rc;
        if ((rc = c->cuda(cudaStreamSynchronize(c->stream), "prepare fast"))) return rc;
        F.scene_key = c->scene_version;
    }
    if (F.has_volumes)
        return c->fail(AE_ERR_STATE, "participating media consume RNG in the reference's visit order; use the plain kernel");
    c->fast_ready = true;
    return AE_OK;
}

void destroy_fast(Ctx *c) {
    delete c->fast;
    c->fast = nullptr;
}

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
AE_DEV bool tri_test_wt(f3 o, const WtRay &W, float tn, float tf, const float4 &r0, const float4 &r1,
                        const float4 &r2, float &t, float &a, float &b) {
    const f3 A = mk(r0.x, r0.y, r0.z) - o, B = mk(r0.w, r1.x, r1.y) - o, C = mk(r1.z, r1.w, r2.x) - o;
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

// Entry distance of the 4 quantised child boxes; an inverted slot or a miss
// yields +inf.  Computed as q * (s/d) + (o - p)/d per slab with a relative
// widening of 2^-20 on the exit side, which covers the rounding of this
// formulation (the decoded boxes already contain the exact ones).
AE_DEV void child_hits(const QNode *nodep, f3 o, f3 inv, float tn, float tf, float tmin[4], uint32_t child[4]) {
    const float4 *p = reinterpret_cast<const float4 *>(nodep);
    const float4 w0 = __ldg(p), w1 = __ldg(p + 1), w2 = __ldg(p + 2), w3 = __ldg(p + 3);
    const uint32_t meta = __float_as_uint(w0.w);
    const int ex = int(int8_t(meta & 0xff)), ey = int(int8_t((meta >> 8) & 0xff)), ez = int(int8_t((meta >> 16) & 0xff));
    const float sx = __int_as_float((ex + 127) << 23), sy = __int_as_float((ey + 127) << 23),
                sz = __int_as_float((ez + 127) << 23);
    const float ix = sx * inv.x, iy = sy * inv.y, iz = sz * inv.z;
    const float bx = (w0.x - o.x) * inv.x, by = (w0.y - o.y) * inv.y, bz = (w0.z - o.z) * inv.z;
    const uint32_t qlo[3] = {__float_as_uint(w1.x), __float_as_uint(w1.y), __float_as_uint(w1.z)};
    const uint32_t qhi[3] = {__float_as_uint(w1.w), __float_as_uint(w2.x), __float_as_uint(w2.y)};
    child[0] = __float_as_uint(w2.z); child[1] = __float_as_uint(w2.w);
    child[2] = __float_as_uint(w3.x); child[3] = __float_as_uint(w3.y);
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const float lx = float((qlo[0] >> (8 * k)) & 0xff), hx = float((qhi[0] >> (8 * k)) & 0xff);
        const float ly = float((qlo[1] >> (8 * k)) & 0xff), hy = float((qhi[1] >> (8 * k)) & 0xff);
        const float lz = float((qlo[2] >> (8 * k)) & 0xff), hz = float((qhi[2] >> (8 * k)) & 0xff);
        const float t0x = fmaf(lx, ix, bx), t1x = fmaf(hx, ix, bx);
        const float t0y = fmaf(ly, iy, by), t1y = fmaf(hy, iy, by);
        const float t0z = fmaf(lz, iz, bz), t1z = fmaf(hz, iz, bz);
        const float lo = fmaxf(fmaxf(fminf(t0x, t1x), fminf(t0y, t1y)), fmaxf(fminf(t0z, t1z), tn));
        const float hi = fminf(fminf(fmaxf(t0x, t1x), fmaxf(t0y, t1y)), fmaxf(t0z, t1z));
        const bool valid = (qlo[0] >> (8 * k) & 0xff) <= (qhi[0] >> (8 * k) & 0xff);
        const bool hit = valid && lo <= fminf(hi * 1.00000095367431640625f, tf);
        tmin[k] = hit ? lo : __int_as_float(0x7f800000);
    }
}

// Safe reciprocal for slab tests: a zero component becomes a huge finite
// value of the same sign, so products stay finite (no 0 * inf).
AE_DEV float slab_inv(float x) { return fabsf(x) > 1e-20f ? 1.0f / x : copysignf(1e20f, x); }

template <bool WT>
AE_DEV void trace_mesh(const FastView &V, const FastInst &I, uint32_t slot, uint64_t orank, f3 o, f3 d, float tn,
                       Best &best, uint2 *stk, int tid, int nthreads) {
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
    uint2 spill[kLocalStack];
    int sp = 0;
    uint32_t cur = I.root;
    for (;;) {
        if (cur & kLeafBit) {
            const uint32_t first = leaf_first(cur), cnt = leaf_count(cur);
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
                    if (sp < kSharedStack) stk[sp * nthreads + tid] = make_uint2(ch[k], __float_as_uint(tm[k]));
                    else if (sp < kFastStack) spill[sp - kSharedStack] = make_uint2(ch[k], __float_as_uint(tm[k]));
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
            const uint2 e = sp < kSharedStack ? stk[sp * nthreads + tid] : spill[sp - kSharedStack];
            if (__uint_as_float(e.y) <= best.t) {
                cur = e.x;
                found = true;
                break;
            }
        }
        if (!found) break;
    }
}

// Closest hit over a ray batch; one thread per ray.  TLAS: the reference's
// binary nodes visited nearest child first; analytic objects use the
// reference intersectors; meshes the 4-wide quantised BLAS.
template <bool WT>
__global__ void __launch_bounds__(128) k_closest_fast(DevScene S, FastView V, const ae_ray *__restrict__ rays,
                                                      uint32_t n, ae_hit *__restrict__ hits) {
    extern __shared__ uint2 stk[];
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int tid = threadIdx.x, nt = blockDim.x;
    const float4 *rp = reinterpret_cast<const float4 *>(rays + i);
    const float4 r0 = __ldg(rp), r1 = __ldg(rp + 1);
    const f3 o = mk(r0.x, r0.y, r0.z), d = mk(r1.x, r1.y, r1.z);
    const float tn = r0.w;
    Best best;
    best.t = kFarStart; best.alpha = 0.0f; best.beta = 0.0f;
    best.object = AE_MISS; best.prim = AE_MISS; best.orank = 0; best.lrank = 0;
    bool any = false;
    if (S.n_nodes > 0) {
        const f3 inv = mk(slab_inv(d.x), slab_inv(d.y), slab_inv(d.z));
        const f3 rinv = 1.0f / d;
        int tstack[kTlasStack];
        float tdist[kTlasStack];
        int sp = 0;
        int cur = 0;
        NodeBox nb = load_node(S.tlas, 0);
        bool live = slab_ref(o, rinv, nb.lo, nb.hi, tn, kFarStart);
        while (live) {
            if (nb.count > 0) {
                const uint32_t first = uint32_t(nb.left);
                for (int k = 0; k < nb.count; k++) {
                    const uint32_t slot = first + uint32_t(k);
                    const uint64_t orank = (uint64_t(~first) << 32) | slot;
                    const uint4 m = __ldg(V.meta + slot);
                    const uint32_t shape = m.x & 0xff;
                    if (shape == AE_SHAPE_MESH) {
                        const float4 *ip = reinterpret_cast<const float4 *>(V.inst + m.y);
                        const float4 a = __ldg(ip), b = __ldg(ip + 1), c = __ldg(ip + 2);
                        FastInst I;
                        I.px = a.x; I.py = a.y; I.pz = a.z; I.scale = a.w;
                        I.qx = b.x; I.qy = b.y; I.qz = b.z; I.qw = b.w;
                        I.root = __float_as_uint(c.x); I.tri_base = __float_as_uint(c.y);
                        trace_mesh<WT>(V, I, slot, orank, o, d, tn, best, stk, tid, nt);
                    } else {
                        DHit h;
                        const ae_object *obj = S.objects + slot;
                        bool hit;
                        if (shape == AE_SHAPE_SPHERE) hit = hit_sphere_ref(obj, o, d, r1.w, tn, best.t, h);
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
                const f3 lt0 = (L.lo - o) * inv, lt1 = (L.hi - o) * inv;
                const f3 rt0 = (R.lo - o) * inv, rt1 = (R.hi - o) * inv;
                const float lmin = fmaxf(fmaxf(fminf(lt0.x, lt1.x), fminf(lt0.y, lt1.y)), fmaxf(fminf(lt0.z, lt1.z), tn));
                const float lmax = fminf(fminf(fmaxf(lt0.x, lt1.x), fmaxf(lt0.y, lt1.y)), fmaxf(lt0.z, lt1.z));
                const float rmin = fmaxf(fmaxf(fminf(rt0.x, rt1.x), fminf(rt0.y, rt1.y)), fmaxf(fminf(rt0.z, rt1.z), tn));
                const float rmax = fminf(fminf(fmaxf(rt0.x, rt1.x), fmaxf(rt0.y, rt1.y)), fmaxf(rt0.z, rt1.z));
                const bool lh = lmin <= fminf(lmax * 1.00000095367431640625f, best.t);
                const bool rh = rmin <= fminf(rmax * 1.00000095367431640625f, best.t);
                if (lh && rh) {
                    const bool lfirst = lmin <= rmin;
                    if (sp < kTlasStack) {
                        tstack[sp] = lfirst ? nb.right : nb.left;
                        tdist[sp] = lfirst ? rmin : lmin;
                        sp++;
                    }
                    cur = lfirst ? nb.left : nb.right;
                    nb = lfirst ? L : R;
                    continue;
                }
                if (lh) { cur = nb.left; nb = L; continue; }
                if (rh) { cur = nb.right; nb = R; continue; }
            }
            live = false;
            while (sp > 0) {
                sp--;
                if (tdist[sp] <= best.t) {
                    cur = tstack[sp];
                    nb = load_node(S.tlas, uint32_t(cur));
                    live = true;
                    break;
                }
            }
        }
        any = best.object != AE_MISS;
    }
    ae_hit out;
    out.t = any ? best.t : 0.0f;
    out.alpha = any ? best.alpha : 0.0f;
    out.beta = any ? best.beta : 0.0f;
    out.object = best.object;
    out.prim = best.prim;
    hits[i] = out;
}

cudaError_t launch_closest_fast(Ctx *c, const ae_ray *rays, uint32_t n, ae_hit *hits, bool quant, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    FastScene &F = *c->fast;
    FastView V{F.nodes.ptr, F.tris.ptr, F.inst.ptr, F.obj_meta.ptr};
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
