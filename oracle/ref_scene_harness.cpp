// TEST INFRASTRUCTURE ONLY (oracle).  C entry points over the reference's own
// CPU scene code, compiled from its sources where they lie (see Makefile):
// BuildBVH (scene/bvh.h:275), MeshLibrary::Add (scene/mesh_library.h:91) and
// the world-bounds helpers of scene/shapes.h.  The tests compare the library's
// host builders with these, byte for byte.
#include "texture_stub.h"
#include "scene/bvh.h"
#include "scene/mesh.h"
#include "scene/mesh_library.h"
#include "scene/shapes.h"

#include <cstring>

extern "C" {

// bounds: n x 6 floats; nodes: capacity 2n; order: n.
int aeref_build_bvh(const float *bounds, uint32_t n, BVHNode_GPU *nodes, uint32_t *node_count, uint32_t *order) {
    std::vector<AABB> b(n);
    for (uint32_t i = 0; i < n; i++)
        b[i] = AABB{bounds[6 * i], bounds[6 * i + 1], bounds[6 * i + 2], bounds[6 * i + 3], bounds[6 * i + 4], bounds[6 * i + 5]};
    std::vector<BVHNode_GPU> out;
    std::vector<uint32_t> ord;
    BuildBVH(b, out, ord);
    std::memcpy(nodes, out.data(), out.size() * sizeof(BVHNode_GPU));
    std::memcpy(order, ord.data(), ord.size() * sizeof(uint32_t));
    *node_count = uint32_t(out.size());
    return 0;
}

// One mesh through MeshLibrary::Add.  vertices: nv x 8 floats (p, n, uv);
// indices uint16.  Outputs: the library's flattened vertices/indices/BLAS.
int aeref_mesh_add(const float *vertices, uint32_t nv, const uint16_t *indices, uint32_t ni,
                   Vertex_GPU *out_vertices, uint32_t *out_indices, BVHNode_GPU *out_blas, uint32_t *out_blas_count) {
    std::vector<Vertex> verts(nv);
    for (uint32_t i = 0; i < nv; i++) {
        const float *v = vertices + 8 * i;
        verts[i] = Vertex{v[0], v[1], v[2], 1.0f, 1.0f, 1.0f, v[3], v[4], v[5], v[6], v[7]};
    }
    std::vector<uint16_t> inds(indices, indices + ni);
    // Zero-centred bounds: Mesh::SetVertices subtracts the bounds centre.
    Mesh mesh(verts, inds, AABB{0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f});
    MeshLibrary lib;
    lib.Add(mesh, false);
    std::memcpy(out_vertices, lib.Vertices().data(), lib.Vertices().size() * sizeof(Vertex_GPU));
    std::memcpy(out_indices, lib.Indices().data(), lib.Indices().size() * sizeof(uint32_t));
    std::memcpy(out_blas, lib.BLASNodes().data(), lib.BLASNodes().size() * sizeof(BVHNode_GPU));
    *out_blas_count = uint32_t(lib.BLASNodes().size());
    return 0;
}

// MeshBounds (scene/shapes.h:124-145): position xyz, rotation xyzw, local box.
void aeref_mesh_bounds(const float *pos, const float *rot, const float *local, float *out) {
    TransformComponent t;
    t.position = Point3(pos[0], pos[1], pos[2]);
    t.rotation = Quat<float>(rot[3], rot[0], rot[1], rot[2]);
    MeshComponent m;
    m.localBounds = AABB{local[0], local[1], local[2], local[3], local[4], local[5]};
    const AABB b = MeshBounds(t, m);
    out[0] = b.min_x; out[1] = b.min_y; out[2] = b.min_z;
    out[3] = b.max_x; out[4] = b.max_y; out[5] = b.max_z;
}

// QuadBounds (scene/shapes.h:78-87) and BoxBounds (scene/shapes.h:102-112).
void aeref_quad_bounds(const float *pos, const float *rot, const float *u, const float *v, float *out) {
    TransformComponent t;
    t.position = Point3(pos[0], pos[1], pos[2]);
    t.rotation = Quat<float>(rot[3], rot[0], rot[1], rot[2]);
    QuadComponent q;
    q.u = Vec3<float>(u[0], u[1], u[2]);
    q.v = Vec3<float>(v[0], v[1], v[2]);
    const AABB b = QuadBounds(t, q);
    out[0] = b.min_x; out[1] = b.min_y; out[2] = b.min_z;
    out[3] = b.max_x; out[4] = b.max_y; out[5] = b.max_z;
}
void aeref_box_bounds(const float *pos, const float *rot, const float *half, float *out) {
    TransformComponent t;
    t.position = Point3(pos[0], pos[1], pos[2]);
    t.rotation = Quat<float>(rot[3], rot[0], rot[1], rot[2]);
    BoxComponent bc;
    bc.halfExtent = Vec3<float>(half[0], half[1], half[2]);
    const AABB b = BoxBounds(t, bc);
    out[0] = b.min_x; out[1] = b.min_y; out[2] = b.min_z;
    out[3] = b.max_x; out[4] = b.max_y; out[5] = b.max_z;
}

// MeshLibrary::Add (scene/mesh_library.h:91-159) over uint32 indices.  The
// reference's Add reads the uint16 index list of its Mesh class, which cannot
// address the 262,144 vertices of a 512x512 grid; its four steps are run here
// through the reference's own helpers (AABB::Empty, SurroundPoint,
// Surround2Points, BuildBVH) with only the index type widened.  Outputs: the
// BLAS (capacity 2 * ni / 3 nodes, mesh-relative), the indices in leaf-slot
// order and the local bounds (6 floats).  The vertices are appended verbatim
// (step 1), so the caller keeps its own copy.
int aeref_mesh_add_u32(const Vertex_GPU *v, uint32_t nv, const uint32_t *indices, uint32_t ni,
                       BVHNode_GPU *out_blas, uint32_t *out_blas_count, uint32_t *out_indices, float *out_local) {
    AABB local = AABB::Empty();
    for (uint32_t i = 0; i < nv; i++) local = SurroundPoint(local, v[i].px, v[i].py, v[i].pz);
    out_local[0] = local.min_x; out_local[1] = local.min_y; out_local[2] = local.min_z;
    out_local[3] = local.max_x; out_local[4] = local.max_y; out_local[5] = local.max_z;
    const uint32_t tris = ni / 3;
    std::vector<AABB> tb;
    tb.reserve(tris);
    for (uint32_t t = 0; t < tris; t++) {
        const Vertex_GPU &a = v[indices[3 * t]], &b = v[indices[3 * t + 1]], &c = v[indices[3 * t + 2]];
        const AABB edge = Surround2Points(Point3(a.px, a.py, a.pz), Point3(b.px, b.py, b.pz));
        tb.push_back(SurroundPoint(edge, c.px, c.py, c.pz));
    }
    std::vector<BVHNode_GPU> nodes;
    std::vector<uint32_t> order;
    BuildBVH(tb, nodes, order);
    for (uint32_t k = 0; k < uint32_t(order.size()); k++)
        for (int j = 0; j < 3; j++) out_indices[3 * k + j] = indices[order[k] * 3 + j];
    std::memcpy(out_blas, nodes.data(), nodes.size() * sizeof(BVHNode_GPU));
    *out_blas_count = uint32_t(nodes.size());
    return 0;
}

// One mesh entity's object record through the reference's MeshToGPU
// (scene/shapes.h:286-291 over BaseGPU, 182-214): transform (position xyz,
// rotation xyzw) and material fields.
int aeref_mesh_object(const float *pos, const float *rot, const float *albedo, uint32_t type, float fuzz, float ior,
                      float emission, float density, uint32_t instance_index, Object_GPU *out) {
    TransformComponent t;
    t.position = Point3(pos[0], pos[1], pos[2]);
    t.rotation = Quat<float>(rot[3], rot[0], rot[1], rot[2]);
    Material m;
    m.type = static_cast<MaterialType>(type);
    m.albedo = Color(albedo[0], albedo[1], albedo[2]);
    m.fuzz = fuzz;
    m.ior = ior;
    m.emission = emission;
    m.density = density;
    *out = MeshToGPU(t, m, instance_index);
    return 0;
}

}  // extern "C"
