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

}  // extern "C"
