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
// 1.3M-ray bounce set this took 3.70 -> 3.31 ms.  It keeps every block busy
// to the end of the launch, which suits a launch that has the GPU to itself;
// the smaller launches of the pipelined host-buffer call, which overlap on
// three streams, use the static assignment (lane i: rays i, i + grid size,
// ...), whose blocks retire early and make room for the next launch.
constexpr uint32_t kWalkChunk = 64;
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
            w.start(S, mk(r.ox, r.oy, r.oz), mk(r.dx, r.dy, r.dz), r.tnear, r.time);
        }
        uint32_t iter = 0;
        for (;;) {
            if (!__any_sync(0xffffffffu, active)) break;
            // Only the warp's largest phase group steps (warp_pick_group).
            const uint32_t pick = warp_pick_group(active ? w.group() : 0u, active, iter);
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
                w.start(S, mk(r.ox, r.oy, r.oz), mk(r.dx, r.dy, r.dz), r.tnear, r.time);
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
                w.start(S, mk(r.ox, r.oy, r.oz), mk(r.dx, r.dy, r.dz), r.tnear, r.time);
            }
            cbase += take;
            m = __ballot_sync(0xffffffffu, need);
        }
        if (!__any_sync(0xffffffffu, active)) break;
        // Only the warp's largest phase group steps (warp_pick_group): on the
        // 1080p bounce set 3.31 -> 2.70 ms.
        const uint32_t pick = warp_pick_group(w.group(), active, iter);
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
    FastView V{F.nodes.ptr, F.tris.ptr, F.inst.ptr, F.obj_meta.ptr};
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
    FastView V{F.nodes.ptr, F.tris.ptr, F.inst.ptr, F.obj_meta.ptr};
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
