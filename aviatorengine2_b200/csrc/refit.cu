// refit.cu - moving instances without a rebuild.  The reference rebuilds the
// whole TLAS with SAH and re-uploads every array on each dirty frame
// (RebuildAcceleration, renderer/renderer.cpp:1087-1130).  Here new instance
// transforms are uploaded (48 bytes each) and the device recomputes:
//
//   * each mesh object's world box - MeshBounds, scene/shapes.h:124-145: the
//     eight corners of the mesh's local box through the instance transform;
//   * each TLAS node box bottom-up over the existing topology, as the union of
//     its objects' boxes widened on flat axes exactly as MakeNode does
//     (scene/bvh.h:58-89) - the boxes a rebuild would give this topology;
//   * the object records' current and previous transforms (the motion
//     vectors of ApplyPreviousTransforms, renderer/renderer.cpp:1034-1085).
//
// Hits against a refit tree are the hits against the moved scene; only the
// tree's quality (and the visit order among exactly equal distances) can
// differ from a fresh SAH build.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <tuple>
#include <vector>

#include "context.h"
#include "fast.h"
#include "trace_common.cuh"

namespace ae {

struct Refit {
    DevBuf<ae_instance> inst_in;
    DevBuf<float> raw;            // 6 floats per TLAS node: un-widened box
    DevBuf<float> local_bounds;   // 6 floats per instance: its mesh's local box
    DevBuf<int32_t> level_nodes;  // TLAS node ids grouped by depth, deepest first
    std::vector<int32_t> level_start;
    uint64_t topology_version = ~0ull;
    std::map<std::tuple<uint32_t, uint32_t, uint32_t>, ae_aabb> mesh_box;  // (vertexBase, indexBase, tris)
};

void destroy_refit(Ctx *c) {
    delete c->refit;
    c->refit = nullptr;
}

// One thread per object: mesh objects get a new world box and transform.
__global__ void k_refit_objects(ae_object *objects, uint32_t n_objects, const ae_instance *inst,
                                const float *local_bounds, float *obj_box) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_objects) return;
    ae_object &o = objects[s];
    if (o.shapeType != AE_SHAPE_MESH) return;
    const ae_instance I = inst[o.instanceIndex];
    const float *lb = local_bounds + 6 * o.instanceIndex;
    const bool scaled = I.scale != 0.0f && I.scale != 1.0f;
    float mn[3] = {3.402823466e38f, 3.402823466e38f, 3.402823466e38f};
    float mx[3] = {-3.402823466e38f, -3.402823466e38f, -3.402823466e38f};
    if (lb[0] <= lb[3]) {
        for (int corner = 0; corner < 8; corner++) {
            f3 l = mk((corner & 1) ? lb[3] : lb[0], (corner & 2) ? lb[4] : lb[1], (corner & 4) ? lb[5] : lb[2]);
            if (scaled) l = I.scale * l;
            const f3 w = mk(I.px, I.py, I.pz) + quat_rotate(I.qx, I.qy, I.qz, I.qw, l);
            mn[0] = fminf(mn[0], w.x); mn[1] = fminf(mn[1], w.y); mn[2] = fminf(mn[2], w.z);
            mx[0] = fmaxf(mx[0], w.x); mx[1] = fmaxf(mx[1], w.y); mx[2] = fmaxf(mx[2], w.z);
        }
    }
    float *b = obj_box + 6 * s;
    b[0] = mn[0]; b[1] = mn[1]; b[2] = mn[2]; b[3] = mx[0]; b[4] = mx[1]; b[5] = mx[2];
    // Previous transform = the one being replaced (StorePreviousRotation,
    // scene/shapes.h:176-183: the vector part with w made non-negative).
    o.x2 = o.x; o.y2 = o.y; o.z2 = o.z;
    o.x = I.px; o.y = I.py; o.z = I.pz;
}

// Previous rotation from the instance record being replaced.
__global__ void k_refit_prev_rotation(ae_object *objects, uint32_t n_objects, const ae_instance *old_inst) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_objects) return;
    ae_object &o = objects[s];
    if (o.shapeType != AE_SHAPE_MESH) return;
    const ae_instance I = old_inst[o.instanceIndex];
    const bool neg = I.qw < 0.0f;
    o.prevRotX = neg ? -I.qx : I.qx;
    o.prevRotY = neg ? -I.qy : I.qy;
    o.prevRotZ = neg ? -I.qz : I.qz;
}

// Non-mesh objects keep their stored world box; computed once per topology
// by the host and uploaded with the raw boxes (objects never move here).
__device__ __forceinline__ void widen(float &lo, float &hi) {
    // MakeNode, scene/bvh.h:69-83 (bounds_minimum = 0.0001f, scene/aabb.h:12)
    if (hi - lo < 0.0001f) {
        lo = __fsub_rn(lo, __fmul_rn(0.0001f, 0.5f));
        hi = __fadd_rn(hi, __fmul_rn(0.0001f, 0.5f));
    }
}

// One level of the bottom-up pass; nodes of a level are independent.
__global__ void k_refit_level(ae_bvh_node *nodes, float *raw, const float *obj_box, const int32_t *level,
                              int32_t count) {
    const int32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const int32_t ni = level[k];
    ae_bvh_node &n = nodes[ni];
    float b[6];
    if (n.count > 0) {
        b[0] = b[1] = b[2] = 3.402823466e38f;
        b[3] = b[4] = b[5] = -3.402823466e38f;
        for (int i = 0; i < n.count; i++) {
            const float *o = obj_box + 6 * (n.left + i);
            for (int a = 0; a < 3; a++) { b[a] = fminf(b[a], o[a]); b[3 + a] = fmaxf(b[3 + a], o[3 + a]); }
        }
    } else {
        const float *l = raw + 6 * n.left, *r = raw + 6 * n.right;
        for (int a = 0; a < 3; a++) { b[a] = fminf(l[a], r[a]); b[3 + a] = fmaxf(l[3 + a], r[3 + a]); }
    }
    float *out = raw + 6 * ni;
    for (int a = 0; a < 6; a++) out[a] = b[a];
    float lo[3] = {b[0], b[1], b[2]}, hi[3] = {b[3], b[4], b[5]};
    for (int a = 0; a < 3; a++) widen(lo[a], hi[a]);
    n.min_x = lo[0]; n.min_y = lo[1]; n.min_z = lo[2];
    n.max_x = hi[0]; n.max_y = hi[1]; n.max_z = hi[2];
}

}  // namespace ae

using namespace ae;

namespace ae {
// World box of a non-mesh object as ae_pack_scene computed it.  The packed
// TLAS holds only the union per leaf, so the box is recomputed from the
// object record with the host formulas.
ae_aabb analytic_box(const ae_object &o) {
    ae_entity e;
    std::memset(&e, 0, sizeof(e));
    e.shape = o.shapeType;
    e.position[0] = o.x; e.position[1] = o.y; e.position[2] = o.z;
    e.rotation[3] = 1.0f;
    e.radius = o.radius;
    if (o.shapeType == AE_SHAPE_QUAD || o.shapeType == AE_SHAPE_TRIANGLE) {
        // The record holds the rotated edges; bounds of p, p+u, p+v(, p+u+v).
        e.u[0] = o.u_x; e.u[1] = o.u_y; e.u[2] = o.u_z;
        e.v[0] = o.v_x; e.v[1] = o.v_y; e.v[2] = o.v_z;
    } else if (o.shapeType == AE_SHAPE_BOX) {
        const float h = 0.5f * o.rotation;
        e.rotation[1] = std::sin(h);
        e.rotation[3] = std::cos(h);
        e.half_extent[0] = o.half_x; e.half_extent[1] = o.half_y; e.half_extent[2] = o.half_z;
    }
    ae_aabb b;
    ae_entity_bounds(&e, nullptr, &b);
    return b;
}
}  // namespace ae

extern "C" int ae_refit_instances(ae_ctx *ctx, const ae_instance *instances, uint32_t n) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c) return AE_ERR_INVALID;
    if (!c->scene_uploaded) return c->fail(AE_ERR_STATE, "refit before ae_upload_scene");
    if (n != c->n_instances || (n && !instances))
        return c->fail(AE_ERR_INVALID, "refit expects %u instances, got %u", c->n_instances, n);
    for (uint32_t i = 0; i < n; i++) {
        const ae_instance &a = instances[i], &b = c->host_instances[i];
        if (a.vertexBase != b.vertexBase || a.indexBase != b.indexBase || a.triangleCount != b.triangleCount ||
            a.blasBase != b.blasBase)
            return c->fail(AE_ERR_LAYOUT, "refit: instance %u changed its mesh; upload the scene instead", i);
    }
    static_assert(sizeof(ae_aabb) == 24, "box");
    if (!c->refit) c->refit = new (std::nothrow) Refit();
    if (!c->refit) return c->fail(AE_ERR_OOM, "refit state");
    Refit &R = *c->refit;
    const uint32_t nn = c->n_nodes, no = c->n_objects;
    int rc;
    if (R.topology_version != c->scene_version_layout) {
        // Per topology: node levels (deepest first), mesh local boxes.
        std::vector<int32_t> depth(nn, 0), order;
        for (uint32_t i = 0; i < nn; i++) {
            const ae_bvh_node &nd = c->host_tlas[i];
            if (nd.count <= 0) {
                depth[nd.left] = depth[i] + 1;
                depth[nd.right] = depth[i] + 1;
            }
        }
        int maxd = 0;
        for (uint32_t i = 0; i < nn; i++) maxd = std::max(maxd, depth[i]);
        R.level_start.assign(1, 0);
        for (int d = maxd; d >= 0; d--) {
            for (uint32_t i = 0; i < nn; i++)
                if (depth[i] == d) order.push_back(int32_t(i));
            R.level_start.push_back(int32_t(order.size()));
        }
        std::vector<float> lb(size_t(std::max(n, 1u)) * 6, 0.0f);
        for (uint32_t i = 0; i < n; i++) {
            const ae_instance &m = c->host_instances[i];
            const auto key = std::make_tuple(m.vertexBase, m.indexBase, m.triangleCount);
            auto it = R.mesh_box.find(key);
            if (it == R.mesh_box.end()) {
                ae_aabb b{3.402823466e38f, 3.402823466e38f, 3.402823466e38f, -3.402823466e38f, -3.402823466e38f,
                          -3.402823466e38f};
                for (uint64_t k = m.indexBase; k < uint64_t(m.indexBase) + 3ull * m.triangleCount; k++) {
                    const ae_vertex &v = c->host_vertices[m.vertexBase + c->host_indices[k]];
                    b.min_x = std::min(b.min_x, v.px); b.min_y = std::min(b.min_y, v.py); b.min_z = std::min(b.min_z, v.pz);
                    b.max_x = std::max(b.max_x, v.px); b.max_y = std::max(b.max_y, v.py); b.max_z = std::max(b.max_z, v.pz);
                }
                it = R.mesh_box.emplace(key, b).first;
            }
            std::memcpy(&lb[6 * i], &it->second, 24);
        }
        // Boxes of objects that do not move: analytic shapes.
        std::vector<float> ob(size_t(std::max(no, 1u)) * 6, 0.0f);
        for (uint32_t s = 0; s < no; s++) {
            if (c->host_objects[s].shapeType == AE_SHAPE_MESH) continue;
            const ae_aabb b = analytic_box(c->host_objects[s]);
            std::memcpy(&ob[6 * s], &b, 24);
        }
        if (R.raw.reserve(size_t(std::max(nn, 1u)) * 6) || R.local_bounds.reserve(lb.size()) ||
            R.level_nodes.reserve(std::max<size_t>(order.size(), 1)) || R.inst_in.reserve(std::max(n, 1u)) ||
            c->obj_box.reserve(ob.size()))
            return c->fail(AE_ERR_OOM, "refit buffers");
        if ((rc = c->cuda(cudaMemcpyAsync(R.local_bounds.ptr, lb.data(), lb.size() * 4, cudaMemcpyHostToDevice, c->stream),
                          "upload")) ||
            (rc = c->cuda(cudaMemcpyAsync(R.level_nodes.ptr, order.data(), order.size() * 4, cudaMemcpyHostToDevice,
                                          c->stream), "upload")) ||
            (rc = c->cuda(cudaMemcpyAsync(c->obj_box.ptr, ob.data(), ob.size() * 4, cudaMemcpyHostToDevice, c->stream),
                          "upload")))
            return rc;
        R.topology_version = c->scene_version_layout;
    }
    if (n == 0 || nn == 0) return AE_OK;
    if ((rc = c->cuda(cudaMemcpyAsync(R.inst_in.ptr, instances, size_t(n) * sizeof(ae_instance), cudaMemcpyHostToDevice,
                                      c->stream), "upload instances")))
        return rc;
    if ((rc = c->timed_begin())) return rc;
    const int T = 256;
    // Previous rotation from the instance buffer before it is replaced.
    k_refit_prev_rotation<<<(no + T - 1) / T, T, 0, c->stream>>>(c->objects.ptr, no, c->instances.ptr);
    k_refit_objects<<<(no + T - 1) / T, T, 0, c->stream>>>(c->objects.ptr, no, R.inst_in.ptr, R.local_bounds.ptr,
                                                          c->obj_box.ptr);
    if ((rc = c->cuda(cudaMemcpyAsync(c->instances.ptr, R.inst_in.ptr, size_t(n) * sizeof(ae_instance),
                                      cudaMemcpyDeviceToDevice, c->stream), "instances")))
        return rc;
    for (size_t l = 0; l + 1 < R.level_start.size(); l++) {
        const int32_t cnt = R.level_start[l + 1] - R.level_start[l];
        if (cnt <= 0) continue;
        k_refit_level<<<(cnt + T - 1) / T, T, 0, c->stream>>>(c->tlas.ptr, R.raw.ptr, c->obj_box.ptr,
                                                             R.level_nodes.ptr + R.level_start[l], cnt);
        c->launches++;
    }
    c->launches += 1;
    if ((rc = c->cuda(cudaGetLastError(), "refit"))) return rc;
    if ((rc = c->timed_end())) return rc;
    // The optimised walk's instance records follow the new transforms.
    std::memcpy(c->host_instances.data(), instances, size_t(n) * sizeof(ae_instance));
    c->scene_version++;
    return AE_OK;
}

// The device copies of the per-frame arrays, as the kernels see them now
// (after refits).  Any pointer may be null.
extern "C" int ae_download_scene(ae_ctx *ctx, ae_object *objects, ae_bvh_node *tlas, ae_instance *instances) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c) return AE_ERR_INVALID;
    if (!c->scene_uploaded) return c->fail(AE_ERR_STATE, "no scene uploaded");
    int rc = AE_OK;
    if (objects && c->n_objects)
        rc = c->cuda(cudaMemcpyAsync(objects, c->objects.ptr, size_t(c->n_objects) * sizeof(ae_object),
                                     cudaMemcpyDeviceToHost, c->stream), "download objects");
    if (!rc && tlas && c->n_nodes)
        rc = c->cuda(cudaMemcpyAsync(tlas, c->tlas.ptr, size_t(c->n_nodes) * sizeof(ae_bvh_node), cudaMemcpyDeviceToHost,
                                     c->stream), "download tlas");
    if (!rc && instances && c->n_instances)
        rc = c->cuda(cudaMemcpyAsync(instances, c->instances.ptr, size_t(c->n_instances) * sizeof(ae_instance),
                                     cudaMemcpyDeviceToHost, c->stream), "download instances");
    if (!rc) rc = c->cuda(cudaStreamSynchronize(c->stream), "download");
    return rc;
}

extern "C" int ae_scene_sizes(const ae_ctx *ctx, uint32_t *n_objects, uint32_t *n_nodes, uint32_t *n_lights,
                              uint32_t *n_instances) {
    const Ctx *c = reinterpret_cast<const Ctx *>(ctx);
    if (!c) return AE_ERR_INVALID;
    if (n_objects) *n_objects = c->n_objects;
    if (n_nodes) *n_nodes = c->n_nodes;
    if (n_lights) *n_lights = c->n_lights;
    if (n_instances) *n_instances = c->n_instances;
    return AE_OK;
}
