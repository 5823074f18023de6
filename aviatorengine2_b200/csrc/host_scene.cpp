// host_scene.cpp - the host side of the acceleration structure: the binned
// SAH builder, the mesh library and TLAS assembly.  These run on the CPU in the
// reference too (scene/bvh.h, scene/mesh_library.h, scene/shapes.h,
// renderer/renderer.cpp) and produce the byte arrays the kernels consume, so
// their output is pinned bit for bit against the reference's own headers
// compiled here (tests/test_host_scene.py).
//
// Compiled with -ffp-contract=off: every float expression below must round
// exactly as the reference's does.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <new>
#include <numeric>
#include <vector>

#include "../../include/ae_b200.h"

namespace {

// scene/aabb.h:12
constexpr float kBoundsMinimum = 0.0001f;
// scene/bvh.h:13, 93, 101
constexpr int kLeafSize = 4;
constexpr int kSahBins = 12;
constexpr int kMaxDepth = 20;

ae_aabb EmptyBox() { return ae_aabb{FLT_MAX, FLT_MAX, FLT_MAX, -FLT_MAX, -FLT_MAX, -FLT_MAX}; }

// Union of two boxes (scene/aabb.h:70-80).  std::min/max, not fmin: the
// reference's comparison semantics are the ones being reproduced.
ae_aabb Union(const ae_aabb &a, const ae_aabb &b) {
    return ae_aabb{std::min(a.min_x, b.min_x), std::min(a.min_y, b.min_y), std::min(a.min_z, b.min_z),
                   std::max(a.max_x, b.max_x), std::max(a.max_y, b.max_y), std::max(a.max_z, b.max_z)};
}
ae_aabb GrowToPoint(const ae_aabb &a, float x, float y, float z) {
    return ae_aabb{std::min(a.min_x, x), std::min(a.min_y, y), std::min(a.min_z, z),
                   std::max(a.max_x, x), std::max(a.max_y, y), std::max(a.max_z, z)};
}
float Centre(const ae_aabb &b, int axis) {
    switch (axis) {
    case 0: return (b.min_x + b.max_x) * 0.5f;
    case 1: return (b.min_y + b.max_y) * 0.5f;
    default: return (b.min_z + b.max_z) * 0.5f;
    }
}
// Half surface area; the constant factor cancels in every comparison.
float HalfArea(const ae_aabb &b) {
    const float dx = b.max_x - b.min_x, dy = b.max_y - b.min_y, dz = b.max_z - b.min_z;
    return dx * dy + dy * dz + dz * dx;
}

// A node from a box, widening any axis thinner than kBoundsMinimum so a slab
// test never multiplies 0 by infinity (scene/bvh.h:58-89).
ae_bvh_node Node(const ae_aabb &box, int left, int right, int count) {
    ae_bvh_node n;
    std::memset(&n, 0, sizeof(n));
    n.min_x = box.min_x; n.min_y = box.min_y; n.min_z = box.min_z;
    n.max_x = box.max_x; n.max_y = box.max_y; n.max_z = box.max_z;
    if (n.max_x - n.min_x < kBoundsMinimum) { n.min_x -= kBoundsMinimum * 0.5f; n.max_x += kBoundsMinimum * 0.5f; }
    if (n.max_y - n.min_y < kBoundsMinimum) { n.min_y -= kBoundsMinimum * 0.5f; n.max_y += kBoundsMinimum * 0.5f; }
    if (n.max_z - n.min_z < kBoundsMinimum) { n.min_z -= kBoundsMinimum * 0.5f; n.max_z += kBoundsMinimum * 0.5f; }
    n.left = left; n.right = right; n.count = count;
    return n;
}

// Binned SAH builder.  The tree shape is a contract (leaf slots are triangle
// and object IDs), so the steps follow scene/bvh.h:120-265 exactly: 12 bins
// per axis over the centroid extent, cost = half area x count on each side,
// every node above the leaf size splits, std::partition on the winning plane,
// median fallback.  Implemented iteratively over an explicit work list that
// visits nodes in the same pre-order as the reference's recursion.
class SahBuilder {
public:
    SahBuilder(const ae_aabb *bounds, uint32_t n) : bounds_(bounds), n_(n) {}

    void Build(std::vector<ae_bvh_node> &nodes, std::vector<uint32_t> &order) {
        nodes.clear();
        order.clear();
        if (n_ == 0) return;
        nodes.reserve(size_t(n_) * 2);
        order.reserve(n_);
        std::vector<uint32_t> idx(n_);
        std::iota(idx.begin(), idx.end(), 0u);

        // Pre-order with the left child first: node indices and leaf slots come
        // out in the order the recursive builder assigns them.
        struct Task { int start, end, depth, parent; bool isRight; };
        std::vector<Task> work;
        work.push_back({0, int(n_), 0, -1, false});
        while (!work.empty()) {
            const Task task = work.back();
            work.pop_back();
            const int self = int(nodes.size());
            if (task.parent >= 0) {
                if (task.isRight) nodes[task.parent].right = self;
                else nodes[task.parent].left = self;
            }
            int mid;
            ae_aabb box;
            if (Split(idx, task.start, task.end, task.depth, box, mid)) {
                nodes.push_back(Node(box, -1, -1, 0));
                // Right is pushed first so the left subtree is built first.
                work.push_back({mid, task.end, task.depth + 1, self, true});
                work.push_back({task.start, mid, task.depth + 1, self, false});
            } else {
                const int first = int(order.size());
                for (int i = task.start; i < task.end; i++) order.push_back(idx[i]);
                nodes.push_back(Node(box, first, -1, task.end - task.start));
            }
        }
    }

private:
    int Bin(float c, float cmin, float scale) const {
        return std::min(kSahBins - 1, static_cast<int>((c - cmin) * scale));
    }

    // Returns false for a leaf.  On a split, `mid` is the partition point.
    bool Split(std::vector<uint32_t> &idx, int start, int end, int depth, ae_aabb &box, int &mid) const {
        box = EmptyBox();
        float cmin[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
        float cmax[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        for (int i = start; i < end; i++) {
            const ae_aabb &b = bounds_[idx[i]];
            box = Union(box, b);
            for (int a = 0; a < 3; a++) {
                const float c = Centre(b, a);
                cmin[a] = std::min(cmin[a], c);
                cmax[a] = std::max(cmax[a], c);
            }
        }
        const int count = end - start;
        if (count <= kLeafSize || depth >= kMaxDepth) return false;

        int bestAxis = -1, bestSplit = 0;
        float bestCost = FLT_MAX;
        for (int a = 0; a < 3; a++) {
            const float extent = cmax[a] - cmin[a];
            if (extent <= 0.0f) continue;
            const float scale = static_cast<float>(kSahBins) / extent;
            ae_aabb binBox[kSahBins];
            int binCount[kSahBins] = {};
            for (int b = 0; b < kSahBins; b++) binBox[b] = EmptyBox();
            for (int i = start; i < end; i++) {
                const ae_aabb &p = bounds_[idx[i]];
                const int b = Bin(Centre(p, a), cmin[a], scale);
                binBox[b] = Union(binBox[b], p);
                binCount[b]++;
            }
            float leftCost[kSahBins - 1];
            int leftCount[kSahBins - 1];
            ae_aabb acc = EmptyBox();
            int accCount = 0;
            for (int s = 0; s < kSahBins - 1; s++) {
                acc = Union(acc, binBox[s]);
                accCount += binCount[s];
                leftCount[s] = accCount;
                leftCost[s] = accCount > 0 ? HalfArea(acc) * accCount : 0.0f;
            }
            acc = EmptyBox();
            accCount = 0;
            for (int s = kSahBins - 1; s > 0; s--) {
                acc = Union(acc, binBox[s]);
                accCount += binCount[s];
                if (leftCount[s - 1] == 0 || accCount == 0) continue;
                const float cost = leftCost[s - 1] + HalfArea(acc) * accCount;
                if (cost < bestCost) { bestCost = cost; bestAxis = a; bestSplit = s; }
            }
        }

        mid = start + count / 2;
        if (bestAxis >= 0) {
            const float scale = static_cast<float>(kSahBins) / (cmax[bestAxis] - cmin[bestAxis]);
            const float cm = cmin[bestAxis];
            const int axis = bestAxis, split = bestSplit;
            auto it = std::partition(idx.begin() + start, idx.begin() + end, [&](uint32_t i) {
                return Bin(Centre(bounds_[i], axis), cm, scale) < split;
            });
            mid = int(it - idx.begin());
        }
        if (mid <= start || mid >= end) mid = start + count / 2;
        return true;
    }

    const ae_aabb *bounds_;
    uint32_t n_;
};

// ---------------------------------------------------------------------------
// Quaternion helpers on the host, spelled as math/quat.hpp does.
// ---------------------------------------------------------------------------
struct V3 { float x, y, z; };
V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
V3 operator*(float s, V3 v) { return {s * v.x, s * v.y, s * v.z}; }
V3 Cross(V3 u, V3 v) { return {u.y * v.z - u.z * v.y, u.z * v.x - u.x * v.z, u.x * v.y - u.y * v.x}; }
struct Q { float x, y, z, w; };
// rotate(q, v), math/quat.hpp:211-217
V3 Rotate(Q q, V3 v) {
    const V3 u{q.x, q.y, q.z};
    const V3 t = 2.0f * Cross(u, v);
    return v + q.w * t + Cross(u, t);
}
// YawOf, math/quat.hpp:227-231
float YawOf(Q q) { return 2.0f * std::atan2(q.y, q.w); }
// QuatY via angleAxis, math/quat.hpp:163-167
Q QuatY(float radians) {
    const float half = radians * 0.5f;
    const float s = std::sin(half);
    return Q{0.0f * s, 1.0f * s, 0.0f * s, std::cos(half)};
}
Q ToQ(const float r[4]) { return Q{r[0], r[1], r[2], r[3]}; }

// ShaderRotation, scene/shapes.h:160-171
Q ShaderRotation(uint32_t shape, Q r) {
    switch (shape) {
    case AE_SHAPE_MESH: return r;
    case AE_SHAPE_SPHERE:
    case AE_SHAPE_BOX: return QuatY(YawOf(r));
    default: return Q{0.0f, 0.0f, 0.0f, 1.0f};
    }
}
// StorePreviousRotation, scene/shapes.h:176-183
void StorePreviousRotation(ae_object &o, Q q) {
    if (q.w < 0.0f) q = Q{-q.x, -q.y, -q.z, -q.w};
    o.prevRotX = q.x; o.prevRotY = q.y; o.prevRotZ = q.z;
}

bool HasScale(float s) { return s != 0.0f && s != 1.0f; }

}  // namespace

extern "C" {
static int pack_entity(const ae_entity &e, const ae_mesh_library *lib, ae_object &o, ae_instance &inst);
}

namespace ae {
// The device part of MeshLibrary::Add (bvh_build.cu).
int gpu_mesh_blas(const ae_vertex *v, uint32_t nv, const uint32_t *idx, uint32_t ni, ae_bvh_node *out_nodes,
                  uint32_t *out_count, uint32_t *out_indices);
int gpu_mesh_blas_many_host(uint32_t k, const ae_vertex *const *v, const uint32_t *nv, const uint32_t *const *idx,
                            const uint32_t *ni, ae_bvh_node *const *out_nodes, uint32_t *out_counts,
                            uint32_t *const *out_indices);
}  // namespace ae

// ---------------------------------------------------------------------------
// Mesh library
// ---------------------------------------------------------------------------
struct ae_mesh_library {
    std::vector<ae_vertex> vertices;
    std::vector<uint32_t> indices;
    std::vector<ae_bvh_node> blas;
    std::vector<ae_mesh_range> ranges;
};

extern "C" {

int ae_build_bvh(const ae_aabb *bounds, uint32_t n, ae_bvh_node *out_nodes, uint32_t *out_node_count,
                 uint32_t *out_order) {
    if (!out_node_count || (n > 0 && (!bounds || !out_nodes || !out_order))) return AE_ERR_INVALID;
    std::vector<ae_bvh_node> nodes;
    std::vector<uint32_t> order;
    try {
        SahBuilder(bounds, n).Build(nodes, order);
    } catch (const std::bad_alloc &) {
        return AE_ERR_OOM;
    }
    if (!nodes.empty()) std::memcpy(out_nodes, nodes.data(), nodes.size() * sizeof(ae_bvh_node));
    if (!order.empty()) std::memcpy(out_order, order.data(), order.size() * sizeof(uint32_t));
    *out_node_count = uint32_t(nodes.size());
    return AE_OK;
}

ae_mesh_library *ae_mesh_library_create(void) { return new (std::nothrow) ae_mesh_library(); }
void ae_mesh_library_destroy(ae_mesh_library *lib) { delete lib; }

// MeshLibrary::Add, scene/mesh_library.h:91-159.  With on_gpu the triangle
// boxes, the BLAS and the leaf-order indices come from the device builder
// (bvh_build.cu), which produces the same bytes.
static int mesh_library_add(ae_mesh_library *lib, const ae_vertex *v, uint32_t nv, const uint32_t *idx, uint32_t ni,
                            int double_sided, bool on_gpu) {
    if (!lib || (nv && !v) || (ni && !idx) || ni % 3 != 0) return AE_ERR_INVALID;
    for (uint32_t i = 0; i < ni; i++)
        if (idx[i] >= nv) return AE_ERR_LAYOUT;
    try {
        ae_mesh_range range{};
        range.vertexBase = uint32_t(lib->vertices.size());
        range.indexBase = uint32_t(lib->indices.size());
        range.blasBase = uint32_t(lib->blas.size());
        range.doubleSided = double_sided ? 1u : 0u;
        ae_aabb local = EmptyBox();
        lib->vertices.reserve(lib->vertices.size() + nv);
        for (uint32_t i = 0; i < nv; i++) {
            lib->vertices.push_back(v[i]);
            local = GrowToPoint(local, v[i].px, v[i].py, v[i].pz);
        }
        range.localBounds = local;
        const uint32_t tris = ni / 3;
        range.triangleCount = tris;
        if (on_gpu) {
            std::vector<ae_bvh_node> nodes(size_t(tris) * 2);
            std::vector<uint32_t> leaf_order_indices(ni);
            uint32_t count = 0;
            const int rc = ae::gpu_mesh_blas(v, nv, idx, ni, nodes.data(), &count, leaf_order_indices.data());
            if (rc != AE_OK) return rc;
            lib->indices.insert(lib->indices.end(), leaf_order_indices.begin(), leaf_order_indices.end());
            lib->blas.insert(lib->blas.end(), nodes.begin(), nodes.begin() + count);
            lib->ranges.push_back(range);
            return int(lib->ranges.size() - 1);
        }
        std::vector<ae_aabb> triBounds(tris);
        for (uint32_t t = 0; t < tris; t++) {
            const ae_vertex &a = v[idx[3 * t]], &b = v[idx[3 * t + 1]], &c = v[idx[3 * t + 2]];
            // Surround2Points(a, b) then SurroundPoint(c), scene/aabb.h:96-103
            ae_aabb e{std::min(a.px, b.px), std::min(a.py, b.py), std::min(a.pz, b.pz),
                      std::max(a.px, b.px), std::max(a.py, b.py), std::max(a.pz, b.pz)};
            triBounds[t] = GrowToPoint(e, c.px, c.py, c.pz);
        }
        std::vector<ae_bvh_node> nodes;
        std::vector<uint32_t> order;
        SahBuilder(triBounds.data(), tris).Build(nodes, order);
        // Indices in leaf-slot order: a leaf addresses triangles by slot.
        lib->indices.reserve(lib->indices.size() + ni);
        for (uint32_t slot : order) {
            lib->indices.push_back(idx[slot * 3 + 0]);
            lib->indices.push_back(idx[slot * 3 + 1]);
            lib->indices.push_back(idx[slot * 3 + 2]);
        }
        lib->blas.insert(lib->blas.end(), nodes.begin(), nodes.end());
        lib->ranges.push_back(range);
    } catch (const std::bad_alloc &) {
        return AE_ERR_OOM;
    }
    return int(lib->ranges.size() - 1);
}

int ae_mesh_library_add(ae_mesh_library *lib, const ae_vertex *v, uint32_t nv, const uint32_t *idx, uint32_t ni,
                        int double_sided) {
    return mesh_library_add(lib, v, nv, idx, ni, double_sided, false);
}
int ae_mesh_library_add_gpu(ae_mesh_library *lib, const ae_vertex *v, uint32_t nv, const uint32_t *idx, uint32_t ni,
                            int double_sided) {
    return mesh_library_add(lib, v, nv, idx, ni, double_sided, true);
}

// k calls of ae_mesh_library_add_gpu in one: the k BLAS are built together
// on the GPU (one forest build, bvh_build.cu) and appended in order, each
// exactly as its own call would append it.  out_handles[m] receives mesh m's
// handle; nothing is appended when any mesh is refused.
int ae_mesh_library_add_many_gpu(ae_mesh_library *lib, uint32_t k, const ae_vertex *const *v, const uint32_t *nv,
                                 const uint32_t *const *idx, const uint32_t *ni, const int *double_sided,
                                 int *out_handles) {
    if (!lib || (k && (!v || !nv || !idx || !ni || !out_handles))) return AE_ERR_INVALID;
    for (uint32_t m = 0; m < k; m++) {
        if ((nv[m] && !v[m]) || (ni[m] && !idx[m]) || ni[m] % 3 != 0) return AE_ERR_INVALID;
        for (uint32_t i = 0; i < ni[m]; i++)
            if (idx[m][i] >= nv[m]) return AE_ERR_LAYOUT;
    }
    try {
        std::vector<std::vector<ae_bvh_node>> nodes(k);
        std::vector<std::vector<uint32_t>> leaf_order(k);
        std::vector<ae_bvh_node *> np(k);
        std::vector<uint32_t *> ip(k);
        std::vector<uint32_t> counts(k, 0);
        for (uint32_t m = 0; m < k; m++) {
            nodes[m].resize(std::max<size_t>(size_t(ni[m] / 3) * 2, 1));
            leaf_order[m].resize(std::max<size_t>(ni[m], 1));
            np[m] = nodes[m].data();
            ip[m] = leaf_order[m].data();
        }
        if (k) {
            const int rc = ae::gpu_mesh_blas_many_host(k, v, nv, idx, ni, np.data(), counts.data(), ip.data());
            if (rc != AE_OK) return rc;
        }
        for (uint32_t m = 0; m < k; m++) {
            ae_mesh_range range{};
            range.vertexBase = uint32_t(lib->vertices.size());
            range.indexBase = uint32_t(lib->indices.size());
            range.blasBase = uint32_t(lib->blas.size());
            range.doubleSided = double_sided && double_sided[m] ? 1u : 0u;
            ae_aabb local = EmptyBox();
            lib->vertices.reserve(lib->vertices.size() + nv[m]);
            for (uint32_t i = 0; i < nv[m]; i++) {
                lib->vertices.push_back(v[m][i]);
                local = GrowToPoint(local, v[m][i].px, v[m][i].py, v[m][i].pz);
            }
            range.localBounds = local;
            range.triangleCount = ni[m] / 3;
            lib->indices.insert(lib->indices.end(), leaf_order[m].begin(), leaf_order[m].begin() + ni[m]);
            lib->blas.insert(lib->blas.end(), nodes[m].begin(), nodes[m].begin() + counts[m]);
            lib->ranges.push_back(range);
            out_handles[m] = int(lib->ranges.size() - 1);
        }
    } catch (const std::bad_alloc &) {
        return AE_ERR_OOM;
    }
    return AE_OK;
}

int ae_mesh_library_range(const ae_mesh_library *lib, uint32_t handle, ae_mesh_range *out) {
    if (!lib || !out || handle >= lib->ranges.size()) return AE_ERR_INVALID;
    *out = lib->ranges[handle];
    return AE_OK;
}
void ae_mesh_library_sizes(const ae_mesh_library *lib, uint64_t *nv, uint64_t *ni, uint64_t *nb) {
    if (nv) *nv = lib ? lib->vertices.size() : 0;
    if (ni) *ni = lib ? lib->indices.size() : 0;
    if (nb) *nb = lib ? lib->blas.size() : 0;
}
const ae_vertex *ae_mesh_library_vertices(const ae_mesh_library *lib) { return lib ? lib->vertices.data() : nullptr; }
const uint32_t *ae_mesh_library_indices(const ae_mesh_library *lib) { return lib ? lib->indices.data() : nullptr; }
const ae_bvh_node *ae_mesh_library_blas(const ae_mesh_library *lib) { return lib ? lib->blas.data() : nullptr; }

// World bounds per shape, scene/shapes.h:70-145.
int ae_entity_bounds(const ae_entity *e, const ae_mesh_library *lib, ae_aabb *out) {
    if (!e || !out) return AE_ERR_INVALID;
    const V3 p{e->position[0], e->position[1], e->position[2]};
    const Q q = ToQ(e->rotation);
    switch (e->shape) {
    case AE_SHAPE_SPHERE: {
        const float r = e->radius;
        *out = ae_aabb{p.x - r, p.y - r, p.z - r, p.x + r, p.y + r, p.z + r};
        return AE_OK;
    }
    case AE_SHAPE_QUAD: {
        const V3 u = Rotate(q, V3{e->u[0], e->u[1], e->u[2]});
        const V3 v = Rotate(q, V3{e->v[0], e->v[1], e->v[2]});
        const V3 puv = p + u + v, pu = p + u, pv = p + v;
        const ae_aabb d1{std::min(p.x, puv.x), std::min(p.y, puv.y), std::min(p.z, puv.z),
                         std::max(p.x, puv.x), std::max(p.y, puv.y), std::max(p.z, puv.z)};
        const ae_aabb d2{std::min(pu.x, pv.x), std::min(pu.y, pv.y), std::min(pu.z, pv.z),
                         std::max(pu.x, pv.x), std::max(pu.y, pv.y), std::max(pu.z, pv.z)};
        *out = Union(d1, d2);
        return AE_OK;
    }
    case AE_SHAPE_TRIANGLE: {
        const V3 u = Rotate(q, V3{e->u[0], e->u[1], e->u[2]});
        const V3 v = Rotate(q, V3{e->v[0], e->v[1], e->v[2]});
        const V3 pu = p + u;
        const ae_aabb b{std::min(p.x, pu.x), std::min(p.y, pu.y), std::min(p.z, pu.z),
                        std::max(p.x, pu.x), std::max(p.y, pu.y), std::max(p.z, pu.z)};
        *out = GrowToPoint(b, p.x + v.x, p.y + v.y, p.z + v.z);
        return AE_OK;
    }
    case AE_SHAPE_BOX: {
        const float yaw = YawOf(q);
        const float s = std::fabs(std::sin(yaw)), c = std::fabs(std::cos(yaw));
        const float hx = e->half_extent[0], hy = e->half_extent[1], hz = e->half_extent[2];
        const float ex = c * hx + s * hz, ez = s * hx + c * hz;
        *out = ae_aabb{p.x - ex, p.y - hy, p.z - ez, p.x + ex, p.y + hy, p.z + ez};
        return AE_OK;
    }
    case AE_SHAPE_MESH: {
        if (!lib || e->mesh >= lib->ranges.size()) return AE_ERR_LAYOUT;
        const ae_aabb &b = lib->ranges[e->mesh].localBounds;
        if (b.min_x > b.max_x) { *out = EmptyBox(); return AE_OK; }
        const bool scaled = HasScale(e->scale);
        ae_aabb w = EmptyBox();
        for (int corner = 0; corner < 8; corner++) {
            V3 l{(corner & 1) ? b.max_x : b.min_x, (corner & 2) ? b.max_y : b.min_y, (corner & 4) ? b.max_z : b.min_z};
            if (scaled) l = e->scale * l;
            const V3 wp = p + Rotate(q, l);
            w = GrowToPoint(w, wp.x, wp.y, wp.z);
        }
        *out = w;
        return AE_OK;
    }
    default:
        return AE_ERR_INVALID;
    }
}

// RebuildAcceleration minus the upload (renderer/renderer.cpp:1087-1130):
// bounds -> BuildBVH -> slot order -> LightIndices -> PackObjects.
// One entity's object record (BaseGPU and the shape's fields, scene/shapes.h:
// 182-214, 286-291) and, for a mesh, its instance record (PackObjects,
// renderer/renderer.cpp:833-858).  instanceIndex is left 0: it is the
// mesh's rank among meshes in slot order, known only after the build.
static int pack_entity(const ae_entity &e, const ae_mesh_library *lib, ae_object &o, ae_instance &inst) {
    std::memset(&o, 0, sizeof(o));
    std::memset(&inst, 0, sizeof(inst));
    o.x = e.position[0]; o.y = e.position[1]; o.z = e.position[2];
    o.x2 = e.prev_position[0]; o.y2 = e.prev_position[1]; o.z2 = e.prev_position[2];
    StorePreviousRotation(o, ShaderRotation(e.shape, ToQ(e.prev_rotation)));
    o.r = e.albedo[0]; o.g = e.albedo[1]; o.b = e.albedo[2];
    o.fuzz = e.fuzz; o.refraction = e.ior; o.emission = e.emission; o.density = e.density;
    o.shapeType = e.shape; o.colorType = e.material;
    o.textureID = e.texture_id; o.textureTint = e.texture_tint;
    const Q q = ToQ(e.rotation);
    switch (e.shape) {
    case AE_SHAPE_SPHERE:
        o.radius = e.radius;
        o.rotation = YawOf(q);
        break;
    case AE_SHAPE_QUAD:
    case AE_SHAPE_TRIANGLE: {
        const V3 u = Rotate(q, V3{e.u[0], e.u[1], e.u[2]});
        const V3 v = Rotate(q, V3{e.v[0], e.v[1], e.v[2]});
        o.u_x = u.x; o.u_y = u.y; o.u_z = u.z;
        o.v_x = v.x; o.v_y = v.y; o.v_z = v.z;
        break;
    }
    case AE_SHAPE_BOX:
        o.half_x = e.half_extent[0]; o.half_y = e.half_extent[1]; o.half_z = e.half_extent[2];
        o.rotation = YawOf(q);
        break;
    case AE_SHAPE_MESH: {
        if (!lib || e.mesh >= lib->ranges.size()) return AE_ERR_LAYOUT;
        const ae_mesh_range &r = lib->ranges[e.mesh];
        inst.px = e.position[0]; inst.py = e.position[1]; inst.pz = e.position[2];
        inst.scale = HasScale(e.scale) ? e.scale : 0.0f;
        inst.qx = q.x; inst.qy = q.y; inst.qz = q.z; inst.qw = q.w;
        inst.vertexBase = r.vertexBase; inst.indexBase = r.indexBase;
        inst.triangleCount = r.triangleCount; inst.blasBase = r.blasBase;
        break;
    }
    default:
        return AE_ERR_INVALID;
    }
    return AE_OK;
}

int ae_pack_scene(const ae_entity *ents, uint32_t n, const ae_mesh_library *lib, ae_object *out_objects,
                  ae_bvh_node *out_nodes, uint32_t *out_node_count, uint32_t *out_lights,
                  uint32_t *out_light_count, ae_instance *out_instances, uint32_t *out_instance_count,
                  uint32_t *out_order) {
    if (!out_node_count || !out_light_count || !out_instance_count) return AE_ERR_INVALID;
    if (n > 0 && (!ents || !out_objects || !out_nodes || !out_lights || !out_instances || !out_order))
        return AE_ERR_INVALID;
    try {
        std::vector<ae_aabb> bounds(n);
        for (uint32_t i = 0; i < n; i++) {
            const int rc = ae_entity_bounds(&ents[i], lib, &bounds[i]);
            if (rc != AE_OK) return rc;
        }
        std::vector<ae_bvh_node> nodes;
        std::vector<uint32_t> order;
        SahBuilder(bounds.data(), n).Build(nodes, order);
        if (!nodes.empty()) std::memcpy(out_nodes, nodes.data(), nodes.size() * sizeof(ae_bvh_node));
        *out_node_count = uint32_t(nodes.size());
        uint32_t lights = 0, instances = 0;
        for (uint32_t slot = 0; slot < n; slot++) {
            const ae_entity &e = ents[order[slot]];
            out_order[slot] = order[slot];
            if (e.material == AE_MAT_DIFFUSE_LIGHT) out_lights[lights++] = slot;
            ae_object o;
            ae_instance inst;
            const int rc = pack_entity(e, lib, o, inst);
            if (rc != AE_OK) return rc;
            if (e.shape == AE_SHAPE_MESH) {
                o.instanceIndex = instances;
                out_instances[instances++] = inst;
            }
            out_objects[slot] = o;
        }
        *out_light_count = lights;
        *out_instance_count = instances;
    } catch (const std::bad_alloc &) {
        return AE_ERR_OOM;
    }
    return AE_OK;
}

}  // extern "C"

namespace ae {
// Per entity, in entity order: its world box, object and instance records
// (instanceIndex 0) and flags (bit 0 mesh, bit 1 light) - everything of
// RebuildAcceleration that does not depend on the slot order, for the device
// rebuild (ae_rebuild_scene).
int pack_templates(const ae_entity *ents, uint32_t n, const ae_mesh_library *lib, ae_aabb *bounds,
                   ae_object *objects, ae_instance *instances, uint32_t *flags) {
    for (uint32_t i = 0; i < n; i++) {
        int rc = ae_entity_bounds(&ents[i], lib, &bounds[i]);
        if (rc == AE_OK) rc = pack_entity(ents[i], lib, objects[i], instances[i]);
        if (rc != AE_OK) return rc;
        flags[i] = (ents[i].shape == AE_SHAPE_MESH ? 1u : 0u) | (ents[i].material == AE_MAT_DIFFUSE_LIGHT ? 2u : 0u);
    }
    return AE_OK;
}
}  // namespace ae

// RebuildAcceleration + UploadScene (renderer/renderer.cpp:1087-1130,
// 931-1027) with the build and the packing on the GPU.
extern "C" int ae_rebuild_scene(ae_ctx *ctx, const ae_entity *ents, uint32_t n, const ae_mesh_library *lib) {
    if (!ctx || (n && !ents)) return AE_ERR_INVALID;
    try {
        std::vector<ae_object> objects(std::max(n, 1u));
        std::vector<ae_bvh_node> nodes(2 * size_t(n) + 1);
        std::vector<uint32_t> lights(std::max(n, 1u)), order(std::max(n, 1u));
        std::vector<ae_instance> instances(std::max(n, 1u));
        uint32_t nn = 0, nl = 0, ni = 0;
        const int rc = ae_pack_scene_gpu(ents, n, lib, objects.data(), nodes.data(), &nn, lights.data(), &nl,
                                         instances.data(), &ni, order.data());
        if (rc != AE_OK) return rc;
        return ae_upload_scene(ctx, objects.data(), n, nodes.data(), nn, lights.data(), nl, instances.data(), ni);
    } catch (const std::bad_alloc &) {
        return AE_ERR_OOM;
    }
}
